// section.cu -- a DoubleSection with user-defined edges, resident on one GPU.
//
// The reference lets a user subclass EdgeBinary / EdgeUnary (nelson/
// EdgeBinary.h:133-157, nelson/EdgeUnary.h:84-92) and add the edges to a
// DoubleSection (nelson/DoubleSection.hpp:338-365); each edge's update()
// computes its residual and Jacobian blocks, and BaseSection::
// updateHessianBlocks (nelson/BaseSection.cpp:5-86) accumulates J'J and J'r
// into the blocks of U (first section), V (second section, block diagonal)
// and W (U x V).  Here the parameters and the edge code stay the user's, on
// the device: an evaluate callback writes every edge's whitened residual r_e
// and Jacobian blocks J_a, J_b into two device arrays owned by the section
// (fixed per-edge offsets, nl_section_layout), and the section does the rest:
//   * section_assemble_kernel: one thread per row of a U / V / W block or
//     entry of bU / bV, summing its edges' contributions in edge order (lists
//     built at structureReady), so H and b are bit-reproducible and need no
//     atomics; U = sum J_a' J_a (+ J_a' J_b for a U-U edge), V = sum J_v' J_v,
//     W = sum J_u' J_v, b = sum J' r;
//   * chi2 = sum r_e' r_e, a fixed-grid two-level reduction;
//   * the Schur solve of the library (SchurCore: V^-1, W V^-1, S, the tiled
//     Cholesky, back-substitution; FP64 or mixed);
//   * LevenbergMarquardt / GaussNewton on the host (host_lm.cuh), calling the
//     user's oplus (with the increment in user order), backup and rollback.
// Edge kinds: U-V binary, U-U binary, U unary, V unary.  U blocks have 2, 3, 6
// or 9 parameters, V blocks 3.  An edge to a fixed parameter block is the
// unary edge of its variable side (the user's evaluator reads the fixed
// block itself).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "host_lm.cuh"
#include "schur_core.cuh"

namespace nl {
namespace {

// One output row: kind 0 U, 1 V, 2 W (block idx, row r, all its columns), 3 bU,
// 4 bV (parameter block idx, component r); contributions [q0, q1).
struct SecTask {
  int kind, idx, r, q0, q1, pad;
};
// One edge's share of an output: for each column c, sum over k < m of
// A[a + k sa + r] * B[b + k sb + c], A the Jacobian array, B the Jacobian
// array (matrices) or the residuals (vectors, one column).
struct SecContrib {
  long long a, b;
  int sa, sb, m, pad;
};

constexpr int kSecNT = 256;
constexpr int kSecRedCTAs = 296;  // 2 per SM
constexpr int kSecMaxCols = 9;
inline int sec_cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

// One thread per output row: A[.. + r] is read once per residual row and the
// B row (contiguous, up to 9 values) feeds every column.  Each entry's sum
// runs over the contributions in edge order and their rows in order.
template <typename T>
static __global__ void __launch_bounds__(128) section_assemble_kernel(
    const SecTask* __restrict__ tasks, int ntasks, const SecContrib* __restrict__ q, const double* __restrict__ J,
    const double* __restrict__ R, int bu, T* __restrict__ U, int LU, T* __restrict__ V, int LV, T* __restrict__ W,
    int LW, T* __restrict__ bU, T* __restrict__ bV) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntasks) return;
  const SecTask k = tasks[t];
  const double* X = k.kind >= 3 ? R : J;
  const int ncols = k.kind == 0 ? bu : (k.kind <= 2 ? 3 : 1);
  double s[kSecMaxCols];
#pragma unroll
  for (int c = 0; c < kSecMaxCols; c++) s[c] = 0.0;
  for (int i = k.q0; i < k.q1; i++) {
    const SecContrib c = q[i];
    const double* pa = J + c.a + k.r;
    const double* pb = X + c.b;
    for (int row = 0; row < c.m; row++) {
      const double a = pa[(long long)row * c.sa];
      const double* brow = pb + (long long)row * c.sb;
#pragma unroll
      for (int col = 0; col < kSecMaxCols; col++)
        if (col < ncols) s[col] += a * brow[col];
    }
  }
  T* out;
  switch (k.kind) {
    case 0: out = U + (size_t)k.idx * LU + k.r * bu; break;
    case 1: out = V + (size_t)k.idx * LV + k.r * 3; break;
    case 2: out = W + (size_t)k.idx * LW + k.r * 3; break;
    case 3: out = bU + (size_t)k.idx * bu + k.r; break;
    default: out = bV + (size_t)k.idx * 3 + k.r; break;
  }
#pragma unroll
  for (int col = 0; col < kSecMaxCols; col++)
    if (col < ncols) out[col] = (T)s[col];
}

// The rows with long contribution lists (a U block's diagonal rows gather
// every edge of that block): one warp per row, the lanes striding over the
// contributions, the partial rows butterfly-reduced in a fixed order.
constexpr int kSecLongList = 16;
template <typename T>
static __global__ void __launch_bounds__(256) section_assemble_warp_kernel(
    const SecTask* __restrict__ tasks, int ntasks, const SecContrib* __restrict__ q, const double* __restrict__ J,
    const double* __restrict__ R, int bu, T* __restrict__ U, int LU, T* __restrict__ V, int LV, T* __restrict__ W,
    int LW, T* __restrict__ bU, T* __restrict__ bV) {
  const int t = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (t >= ntasks) return;  // the whole warp
  const SecTask k = tasks[t];
  const double* X = k.kind >= 3 ? R : J;
  const int ncols = k.kind == 0 ? bu : (k.kind <= 2 ? 3 : 1);
  double s[kSecMaxCols];
#pragma unroll
  for (int c = 0; c < kSecMaxCols; c++) s[c] = 0.0;
  for (int i = k.q0 + lane; i < k.q1; i += 32) {
    const SecContrib c = q[i];
    const double* pa = J + c.a + k.r;
    const double* pb = X + c.b;
    for (int row = 0; row < c.m; row++) {
      const double a = pa[(long long)row * c.sa];
      const double* brow = pb + (long long)row * c.sb;
#pragma unroll
      for (int col = 0; col < kSecMaxCols; col++)
        if (col < ncols) s[col] += a * brow[col];
    }
  }
#pragma unroll
  for (int col = 0; col < kSecMaxCols; col++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[col] += __shfl_xor_sync(0xffffffffu, s[col], o);
  if (lane != 0) return;
  T* out;
  switch (k.kind) {
    case 0: out = U + (size_t)k.idx * LU + k.r * bu; break;
    case 1: out = V + (size_t)k.idx * LV + k.r * 3; break;
    case 2: out = W + (size_t)k.idx * LW + k.r * 3; break;
    case 3: out = bU + (size_t)k.idx * bu + k.r; break;
    default: out = bV + (size_t)k.idx * 3 + k.r; break;
  }
#pragma unroll
  for (int col = 0; col < kSecMaxCols; col++)
    if (col < ncols) out[col] = (T)s[col];
}

__device__ __forceinline__ double sec_block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w];
  __syncthreads();
  return t;  // valid in thread 0
}

// per-CTA partial sums of r_i^2 (fixed grid for a given length: deterministic)
static __global__ void __launch_bounds__(kSecNT) section_sumsq_kernel(const double* __restrict__ r, long long n,
                                                                      double* __restrict__ part) {
  __shared__ double sh[kSecNT / 32];
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * kSecNT + threadIdx.x; i < n; i += (long long)gridDim.x * kSecNT)
    s += r[i] * r[i];
  s = sec_block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// one warp: lane-strided partials, then a butterfly (a fixed order)
static __global__ void section_sum_kernel(const double* __restrict__ part, int n, double* __restrict__ out) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) s += part[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) *out = s;
}

// per-CTA partials of |delta|^2 and delta . b over (U, V)
template <typename T>
static __global__ void __launch_bounds__(kSecNT) section_dot_kernel(const double* __restrict__ incU,
                                                                    const T* __restrict__ bU, int nu,
                                                                    const double* __restrict__ incV,
                                                                    const T* __restrict__ bV, int nv,
                                                                    double* __restrict__ part) {
  __shared__ double sh[kSecNT / 32];
  double a = 0.0, c = 0.0;
  for (int i = blockIdx.x * kSecNT + threadIdx.x; i < nu + nv; i += gridDim.x * kSecNT) {
    const double x = i < nu ? incU[i] : incV[i - nu];
    const double g = i < nu ? (double)bU[i] : (double)bV[i - nu];
    a += x * x;
    c += x * g;
  }
  a = sec_block_sum(a, sh);
  c = sec_block_sum(c, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = c;
  }
}

// the increment of U in user order: out[u] = inc[perm[u]]
static __global__ void section_user_inc_kernel(const double* __restrict__ inc, const int* __restrict__ perm, int nu,
                                               int bu, double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nu * bu) return;
  const int u = t / bu, i = t - u * bu;
  out[t] = inc[(size_t)perm[u] * bu + i];
}

}  // namespace
}  // namespace nl

using namespace nl;

struct nl_section {
  int bu = 0, nu = 0, nv = 0, precision = NL_PREC_FP64, device = 0;
  bool ready = false;
  cudaStream_t st = nullptr;
  cublasHandle_t cublas = nullptr;
  DevBuf ws, r, jac, tasks, tasks_long, contribs, d_perm, inc_user, scal, lam, part;
  std::unique_ptr<SchurCore> core;
  std::vector<int> kind, ea, eb, em, perm;
  std::vector<long long> r_off{0}, j_off{0};
  std::vector<std::pair<int, int>> ublk;  // U pattern, (col, row) internal, CSC order
  std::vector<std::pair<int, int>> wblk;  // W pattern, (U block internal, V block), CSR order
  int ntasks = 0, ntasks_long = 0;  // rows with short / long contribution lists
  nl_section_callbacks cb{};
  bool have_cb = false;
  double chi2 = 0.0, max_b = 0.0, inc_sq = 0.0, inc_b = 0.0;
  double* pin = nullptr;  // pinned scalars: 0 chi2, 1 max|b|, 2 max|diag H|, 3..4 lam, 5 status
  std::vector<double> dot_part;
  ~nl_section() {
    core.reset();
    if (cublas) cublasDestroy(cublas);
    if (pin) cudaFreeHost(pin);
    if (st) cudaStreamDestroy(st);
  }
  int dim(int k, int side) const { return (k == NL_EDGE_V || (k == NL_EDGE_UV && side == 1)) ? 3 : bu; }
  long long red_grid(long long n) const { return std::max(1, std::min(kSecRedCTAs, sec_cdiv(n, kSecNT))); }
};

namespace {

#define SEC_CUDA(x)                                      \
  do {                                                   \
    if ((x) != cudaSuccess) throw HostError{NL_ERR_CUDA}; \
  } while (0)

// The problem operations of the LM / GN loops (host_lm.cuh) on a section.
struct SectionOps {
  nl_section* h;
  void drain() { SEC_CUDA(cudaStreamSynchronize(h->st)); }
  void call(int rc) {
    if (rc != 0) throw HostError{NL_ERR_CALLBACK};
    SEC_CUDA(cudaGetLastError());
  }
  void update(bool hess) {
    drain();
    call(h->cb.evaluate(h->cb.user, (void*)h->st, hess ? 1 : 0, h->r.as<double>(), h->jac.as<double>()));
    const long long R = h->r_off.back();
    const int g = (int)h->red_grid(R);
    section_sumsq_kernel<<<g, kSecNT, 0, h->st>>>(h->r.as<double>(), R, h->part.as<double>());
    section_sum_kernel<<<1, 32, 0, h->st>>>(h->part.as<double>(), g, h->scal.as<double>());
    SEC_CUDA(cudaGetLastError());
    SEC_CUDA(cudaMemcpyAsync(h->pin, h->scal.p, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    if (hess) {
      const bool f64 = h->precision == NL_PREC_FP64;
      if (h->ntasks + h->ntasks_long > 0) {
#define SEC_ASM(T, BC)                                                                                               \
  do {                                                                                                                \
    if (h->ntasks > 0)                                                                                                \
      section_assemble_kernel<T><<<sec_cdiv(h->ntasks, 128), 128, 0, h->st>>>(                                        \
          h->tasks.as<SecTask>(), h->ntasks, h->contribs.as<SecContrib>(), h->jac.as<double>(), h->r.as<double>(),    \
          h->bu, (T*)h->core->dU(), Layout<T, BC>::U, (T*)h->core->dV(), Layout<T, BC>::V, (T*)h->core->dW(),         \
          Layout<T, BC>::W, (T*)h->core->dbU(), (T*)h->core->dbV());                                                  \
    if (h->ntasks_long > 0)                                                                                           \
      section_assemble_warp_kernel<T><<<sec_cdiv(h->ntasks_long, 8), 256, 0, h->st>>>(                                \
          h->tasks_long.as<SecTask>(), h->ntasks_long, h->contribs.as<SecContrib>(), h->jac.as<double>(),             \
          h->r.as<double>(), h->bu, (T*)h->core->dU(), Layout<T, BC>::U, (T*)h->core->dV(), Layout<T, BC>::V,         \
          (T*)h->core->dW(), Layout<T, BC>::W, (T*)h->core->dbU(), (T*)h->core->dbV());                               \
  } while (0)
        switch (h->bu) {
          case 2: if (f64) SEC_ASM(double, 2); else SEC_ASM(float, 2); break;
          case 3: if (f64) SEC_ASM(double, 3); else SEC_ASM(float, 3); break;
          case 6: if (f64) SEC_ASM(double, 6); else SEC_ASM(float, 6); break;
          default: if (f64) SEC_ASM(double, 9); else SEC_ASM(float, 9); break;
        }
#undef SEC_ASM
        SEC_CUDA(cudaGetLastError());
      }
      host_check(h->core->enqueue_maxabs_b(h->scal.as<double>() + 1, nullptr));
      SEC_CUDA(cudaMemcpyAsync(h->pin + 1, h->scal.as<double>() + 1, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    }
    drain();
    h->chi2 = h->pin[0];
    if (hess) h->max_b = h->pin[1];
  }
  double chi2() const { return h->chi2; }
  double max_abs_b() const { return h->max_b; }
  double max_abs_hdiag() {
    host_check(h->core->enqueue_hdiag(h->scal.as<double>() + 2));
    SEC_CUDA(cudaMemcpyAsync(h->pin + 2, h->scal.as<double>() + 2, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    drain();
    return h->pin[2];
  }
  bool compute_increment(double rel, double abs_) {
    h->pin[3] = rel;
    h->pin[4] = abs_;
    SEC_CUDA(cudaMemcpyAsync(h->lam.p, h->pin + 3, 2 * sizeof(double), cudaMemcpyHostToDevice, h->st));
    int* status = reinterpret_cast<int*>(h->lam.as<double>() + 2);
    SEC_CUDA(cudaMemsetAsync(status, 0, sizeof(int), h->st));
    host_check(h->core->enqueue_increment(h->lam.as<double>(), status, nullptr));
    const int nuu = h->nu * h->bu, nvv = 3 * h->nv;
    const int g = (int)h->red_grid(nuu + nvv);
    if (h->precision == NL_PREC_FP64)
      section_dot_kernel<double><<<g, kSecNT, 0, h->st>>>(h->core->incU, (const double*)h->core->dbU(), nuu,
                                                          h->core->incV, (const double*)h->core->dbV(), nvv,
                                                          h->part.as<double>());
    else
      section_dot_kernel<float><<<g, kSecNT, 0, h->st>>>(h->core->incU, (const float*)h->core->dbU(), nuu,
                                                         h->core->incV, (const float*)h->core->dbV(), nvv,
                                                         h->part.as<double>());
    SEC_CUDA(cudaGetLastError());
    h->dot_part.resize(2 * (size_t)g);
    SEC_CUDA(cudaMemcpyAsync(h->dot_part.data(), h->part.p, sizeof(double) * 2 * g, cudaMemcpyDeviceToHost, h->st));
    SEC_CUDA(cudaMemcpyAsync(h->pin + 5, status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    drain();
    double a = 0.0, c = 0.0;
    for (int i = 0; i < g; i++) {
      a += h->dot_part[2 * i];
      c += h->dot_part[2 * i + 1];
    }
    h->inc_sq = a;
    h->inc_b = c;
    int stt = 0;
    memcpy(&stt, h->pin + 5, sizeof(int));
    if (stt & ST_SPIN_TIMEOUT) throw HostError{NL_ERR_TIMEOUT};
    return stt == 0;
  }
  double inc_sqnorm() const { return h->inc_sq; }
  // computeRhoChi2Change (nelson/DoubleSection.h:300-311) with the candidate's
  // chi2 already evaluated: (old - new) / delta' (mu delta - b)
  double rho(double mu, double oldChi2) const { return (oldChi2 - h->chi2) / (mu * h->inc_sq - h->inc_b); }
  void oplus() {
    const int n = h->nu * h->bu;
    if (n > 0) {
      section_user_inc_kernel<<<sec_cdiv(n, 256), 256, 0, h->st>>>(h->core->incU, h->d_perm.as<int>(), h->nu, h->bu,
                                                                   h->inc_user.as<double>());
      SEC_CUDA(cudaGetLastError());
    }
    drain();
    call(h->cb.oplus(h->cb.user, (void*)h->st, h->inc_user.as<double>(), h->core->incV));
  }
  void backup() {
    if (!h->cb.backup) throw HostError{NL_ERR_STATE};
    drain();
    call(h->cb.backup(h->cb.user, (void*)h->st));
  }
  void rollback() {
    if (!h->cb.rollback) throw HostError{NL_ERR_STATE};
    drain();
    call(h->cb.rollback(h->cb.user, (void*)h->st));
  }
};

}  // namespace

extern "C" {

nl_status nl_section_create(int bu, int nu, int nv, int precision, int device, nl_section** out) {
  if (!out || nu < 1 || nv < 0 || (bu != 2 && bu != 3 && bu != 6 && bu != 9) ||
      (precision != NL_PREC_FP64 && precision != NL_PREC_MIXED))
    return NL_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<nl_section> h(new nl_section());
  h->bu = bu;
  h->nu = nu;
  h->nv = nv;
  h->precision = precision;
  h->device = device;
  h->perm.resize(nu);
  for (int i = 0; i < nu; i++) h->perm[i] = i;
  NL_CUDA(cudaSetDevice(device));
  NL_CUDA(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  NL_CUDA(cudaMallocHost(&h->pin, 64));
  *out = h.release();
  return NL_OK;
}

nl_status nl_section_destroy(nl_section* s) {
  if (!s) return NL_ERR_ARG;
  cudaSetDevice(s->device);
  if (s->st) cudaStreamSynchronize(s->st);
  delete s;
  return NL_OK;
}

// DoubleSection::addEdge for n user edges; every index and size is checked
// before any is kept
nl_status nl_section_add_edges(nl_section* s, int n, const int* kind, const int* a, const int* b, const int* m) {
  if (!s || s->ready || n < 0 || (n > 0 && (!kind || !a || !m))) return NL_ERR_ARG;
  for (int e = 0; e < n; e++) {
    const int k = kind[e];
    if (m[e] < 1 || m[e] > 64) return NL_ERR_ARG;
    switch (k) {
      case NL_EDGE_UV:
        if (!b || a[e] < 0 || a[e] >= s->nu || b[e] < 0 || b[e] >= s->nv) return NL_ERR_ARG;
        break;
      case NL_EDGE_UU:
        if (!b || a[e] < 0 || a[e] >= s->nu || b[e] < 0 || b[e] >= s->nu || a[e] == b[e]) return NL_ERR_ARG;
        break;
      case NL_EDGE_U:
        if (a[e] < 0 || a[e] >= s->nu) return NL_ERR_ARG;
        break;
      case NL_EDGE_V:
        if (a[e] < 0 || a[e] >= s->nv) return NL_ERR_ARG;
        break;
      default:
        return NL_ERR_ARG;
    }
  }
  for (int e = 0; e < n; e++) {
    const int k = kind[e];
    const bool binary = k == NL_EDGE_UV || k == NL_EDGE_UU;
    s->kind.push_back(k);
    s->ea.push_back(a[e]);
    s->eb.push_back(binary ? b[e] : -1);
    s->em.push_back(m[e]);
    const long long cols = s->dim(k, 0) + (binary ? s->dim(k, 1) : 0);
    s->r_off.push_back(s->r_off.back() + m[e]);
    s->j_off.push_back(s->j_off.back() + (long long)m[e] * cols);
  }
  return NL_OK;
}

nl_status nl_section_set_user2internal_u(nl_section* s, const int* perm) {
  if (!s || !perm || s->ready) return NL_ERR_ARG;
  std::vector<char> seen(s->nu, 0);
  for (int i = 0; i < s->nu; i++) {
    if (perm[i] < 0 || perm[i] >= s->nu || seen[perm[i]]) return NL_ERR_ARG;
    seen[perm[i]] = 1;
  }
  std::copy(perm, perm + s->nu, s->perm.begin());
  return NL_OK;
}

// permuteAMD_SchurU (nelson/DoubleSection.hpp:30-63): approximate minimum
// degree of the pattern of U + W W'.  A U-V edge joins its U block to the V
// block's clique; a U-U edge is a two-block clique of its own.
nl_status nl_section_permute_amd_u(nl_section* s) {
  if (!s || s->ready) return NL_ERR_ARG;
  std::vector<int> cam, pt;
  int extra = 0;
  for (size_t e = 0; e < s->kind.size(); e++) {
    if (s->kind[e] == NL_EDGE_UV) {
      cam.push_back(s->ea[e]);
      pt.push_back(s->eb[e]);
    } else if (s->kind[e] == NL_EDGE_UU) {
      cam.push_back(s->ea[e]);
      pt.push_back(s->nv + extra);
      cam.push_back(s->eb[e]);
      pt.push_back(s->nv + extra);
      extra++;
    }
  }
  return nl_amd_order_camera_graph(s->nu, s->nv + extra, (int)cam.size(), cam.data(), pt.data(), s->perm.data());
}

// DoubleSection::structureReady: the U pattern (all diagonal blocks plus the
// U-U edge pairs, upper CSC in internal order), V (one block per V block), W
// (the U-V edge pairs, CSR), each output entry's contribution list in edge
// order, device buffers, the Schur solver.
nl_status nl_section_structure_ready(nl_section* s) {
  if (!s || s->ready) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(s->device));
  const int ne = (int)s->kind.size(), bu = s->bu, nu = s->nu, nv = s->nv;
  auto& ublk = s->ublk;
  auto& wblk = s->wblk;
  ublk.clear();
  wblk.clear();
  for (int i = 0; i < nu; i++) ublk.push_back({i, i});
  for (int e = 0; e < ne; e++) {
    if (s->kind[e] == NL_EDGE_UU) {
      const int i = s->perm[s->ea[e]], j = s->perm[s->eb[e]];
      ublk.push_back({std::max(i, j), std::min(i, j)});
    } else if (s->kind[e] == NL_EDGE_UV) {
      wblk.push_back({s->perm[s->ea[e]], s->eb[e]});
    }
  }
  std::sort(ublk.begin(), ublk.end());
  ublk.erase(std::unique(ublk.begin(), ublk.end()), ublk.end());
  std::sort(wblk.begin(), wblk.end());
  wblk.erase(std::unique(wblk.begin(), wblk.end()), wblk.end());
  const int nU = (int)ublk.size(), nW = (int)wblk.size();
  auto uid = [&](int r, int c) {  // block (row r <= col c)
    return (int)(std::lower_bound(ublk.begin(), ublk.end(), std::make_pair(c, r)) - ublk.begin());
  };
  auto wid = [&](int u, int v) {
    return (int)(std::lower_bound(wblk.begin(), wblk.end(), std::make_pair(u, v)) - wblk.begin());
  };
  // contribution lists, in edge order
  std::vector<std::vector<SecContrib>> uq(nU), vq(nv), wq(nW), bq(nu), cq(nv);
  for (int e = 0; e < ne; e++) {
    const int k = s->kind[e], m = s->em[e];
    const long long ja = s->j_off[e], ro = s->r_off[e];
    const int da = s->dim(k, 0);
    const long long jb = ja + (long long)m * da;
    switch (k) {
      case NL_EDGE_UV: {
        const int i = s->perm[s->ea[e]], p = s->eb[e];
        uq[uid(i, i)].push_back({ja, ja, bu, bu, m, 0});
        vq[p].push_back({jb, jb, 3, 3, m, 0});
        wq[wid(i, p)].push_back({ja, jb, bu, 3, m, 0});
        bq[i].push_back({ja, ro, bu, 1, m, 0});
        cq[p].push_back({jb, ro, 3, 1, m, 0});
        break;
      }
      case NL_EDGE_UU: {
        const int i = s->perm[s->ea[e]], j = s->perm[s->eb[e]];
        uq[uid(i, i)].push_back({ja, ja, bu, bu, m, 0});
        uq[uid(j, j)].push_back({jb, jb, bu, bu, m, 0});
        if (i < j)
          uq[uid(i, j)].push_back({ja, jb, bu, bu, m, 0});
        else
          uq[uid(j, i)].push_back({jb, ja, bu, bu, m, 0});
        bq[i].push_back({ja, ro, bu, 1, m, 0});
        bq[j].push_back({jb, ro, bu, 1, m, 0});
        break;
      }
      case NL_EDGE_U: {
        const int i = s->perm[s->ea[e]];
        uq[uid(i, i)].push_back({ja, ja, bu, bu, m, 0});
        bq[i].push_back({ja, ro, bu, 1, m, 0});
        break;
      }
      default: {
        const int p = s->ea[e];
        vq[p].push_back({ja, ja, 3, 3, m, 0});
        cq[p].push_back({ja, ro, 3, 1, m, 0});
        break;
      }
    }
  }
  std::vector<SecContrib> contribs;
  std::vector<SecTask> tasks, tasks_long;
  auto add = [&](int kind, int idx, int rows, int /*cols: all of the row's, in the kernel*/,
                 const std::vector<SecContrib>& l) {
    const int q0 = (int)contribs.size();
    contribs.insert(contribs.end(), l.begin(), l.end());
    const int q1 = (int)contribs.size();
    for (int r = 0; r < rows; r++) (q1 - q0 > kSecLongList ? tasks_long : tasks).push_back({kind, idx, r, q0, q1, 0});
  };
  for (int q = 0; q < nU; q++) add(0, q, bu, bu, uq[q]);
  for (int p = 0; p < nv; p++) add(1, p, 3, 3, vq[p]);
  for (int q = 0; q < nW; q++) add(2, q, bu, 3, wq[q]);
  for (int i = 0; i < nu; i++) add(3, i, bu, 1, bq[i]);
  for (int p = 0; p < nv; p++) add(4, p, 3, 1, cq[p]);
  if (contribs.size() > (size_t)0x7fffffff || tasks.size() > (size_t)0x7fffffff) return NL_ERR_UNSUPPORTED;
  s->ntasks = (int)tasks.size();
  s->ntasks_long = (int)tasks_long.size();
  nl_status st;
  if ((st = upload(s->tasks, tasks, s->st)) != NL_OK) return st;
  if ((st = upload(s->tasks_long, tasks_long, s->st)) != NL_OK) return st;
  if ((st = upload(s->contribs, contribs, s->st)) != NL_OK) return st;
  if ((st = upload(s->d_perm, s->perm, s->st)) != NL_OK) return st;
  if ((st = s->r.alloc(sizeof(double) * (size_t)std::max(s->r_off.back(), 1LL))) != NL_OK) return st;
  if ((st = s->jac.alloc(sizeof(double) * (size_t)std::max(s->j_off.back(), 1LL))) != NL_OK) return st;
  NL_CUDA(cudaMemsetAsync(s->r.p, 0, s->r.bytes, s->st));
  NL_CUDA(cudaMemsetAsync(s->jac.p, 0, s->jac.bytes, s->st));
  if ((st = s->inc_user.alloc(sizeof(double) * (size_t)std::max(nu * bu, 1))) != NL_OK) return st;
  if ((st = s->scal.alloc(64)) != NL_OK) return st;
  if ((st = s->lam.alloc(64)) != NL_OK) return st;
  if ((st = s->part.alloc(sizeof(double) * 2 * kSecRedCTAs)) != NL_OK) return st;
  if (s->precision == NL_PREC_FP64) {
    if (cublasCreate(&s->cublas) != CUBLAS_STATUS_SUCCESS) return NL_ERR_CUDA;
    cublasSetStream(s->cublas, s->st);
    if ((st = s->ws.alloc(64u << 20)) != NL_OK) return st;
    cublasSetWorkspace(s->cublas, s->ws.p, s->ws.bytes);
  }
  s->core = make_schur_core(s->precision, bu, s->cublas);
  if (!s->core) return NL_ERR_UNSUPPORTED;
  s->core->refine_sweeps = s->precision == NL_PREC_MIXED ? 1 : 0;
  s->core->keep_schur = 0;
  s->core->use_tc = s->precision == NL_PREC_MIXED ? 1 : 0;
  SchurStructure ss;
  ss.bc = bu;
  ss.nci = nu;
  ss.np = nv;
  for (auto& b : ublk) {
    ss.u_r.push_back(b.second);
    ss.u_c.push_back(b.first);
  }
  ss.v_uid.resize(nv);
  for (int p = 0; p < nv; p++) ss.v_uid[p] = p;
  for (auto& w : wblk) {
    ss.w_r.push_back(w.first);
    ss.w_c.push_back(w.second);
  }
  if ((st = s->core->setup(ss, s->st)) != NL_OK) return st;
  NL_CUDA(cudaStreamSynchronize(s->st));
  s->ready = true;
  return NL_OK;
}

nl_status nl_section_get_user2internal_u(nl_section* s, int* perm) {
  if (!s || !perm) return NL_ERR_ARG;
  std::copy(s->perm.begin(), s->perm.end(), perm);
  return NL_OK;
}

nl_status nl_section_get_counts(nl_section* s, int* nU, int* nW, long long* r_len, long long* j_len) {
  if (!s) return NL_ERR_ARG;
  if (!s->ready) return NL_ERR_STATE;
  if (nU) *nU = (int)s->ublk.size();
  if (nW) *nW = (int)s->wblk.size();
  if (r_len) *r_len = s->r_off.back();
  if (j_len) *j_len = s->j_off.back();
  return NL_OK;
}

nl_status nl_section_layout(nl_section* s, long long* r_off, long long* j_off) {
  if (!s) return NL_ERR_ARG;
  if (r_off) std::copy(s->r_off.begin(), s->r_off.end(), r_off);
  if (j_off) std::copy(s->j_off.begin(), s->j_off.end(), j_off);
  return NL_OK;
}

nl_status nl_section_get_patterns(nl_section* s, int* u_rc, int* w_rc) {
  if (!s) return NL_ERR_ARG;
  if (!s->ready) return NL_ERR_STATE;
  if (u_rc)
    for (size_t q = 0; q < s->ublk.size(); q++) {
      u_rc[2 * q] = s->ublk[q].second;
      u_rc[2 * q + 1] = s->ublk[q].first;
    }
  if (w_rc)
    for (size_t q = 0; q < s->wblk.size(); q++) {
      w_rc[2 * q] = s->wblk[q].first;
      w_rc[2 * q + 1] = s->wblk[q].second;
    }
  return NL_OK;
}

nl_status nl_section_set_callbacks(nl_section* s, const nl_section_callbacks* cb) {
  if (!s || !cb || !cb->evaluate || !cb->oplus) return NL_ERR_ARG;
  s->cb = *cb;
  s->have_cb = true;
  return NL_OK;
}

nl_status nl_section_set_solver_kind(nl_section* s, int kind) {
  if (!s || !s->ready) return NL_ERR_STATE;
  if (kind != NL_SOLVER_DENSE && kind != NL_SOLVER_ENVELOPE) return NL_ERR_ARG;
  s->core->envelope = kind == NL_SOLVER_ENVELOPE ? 1 : 0;
  return NL_OK;
}

nl_status nl_section_update(nl_section* s, int hessian, double* chi2) {
  if (!s) return NL_ERR_ARG;
  if (!s->ready || !s->have_cb) return NL_ERR_STATE;
  try {
    NL_CUDA(cudaSetDevice(s->device));
    SectionOps P{s};
    P.update(hessian != 0);
    if (chi2) *chi2 = s->chi2;
  } catch (const HostError& e) {
    return e.s;
  }
  return NL_OK;
}

nl_status nl_section_get_hessian(nl_section* s, double* U, double* V, double* W, double* bU, double* bV) {
  if (!s) return NL_ERR_ARG;
  if (!s->ready) return NL_ERR_STATE;
  NL_CUDA(cudaSetDevice(s->device));
  return s->core->get_hessian(U, V, W, bU, bV);
}

nl_status nl_section_compute_increment(nl_section* s, double rel, double abs_, double* incU, double* incV, int* ok) {
  if (!s) return NL_ERR_ARG;
  if (!s->ready) return NL_ERR_STATE;
  try {
    NL_CUDA(cudaSetDevice(s->device));
    SectionOps P{s};
    const bool good = P.compute_increment(rel, abs_);
    const int n = s->nu * s->bu;
    if (incU && n > 0) {
      section_user_inc_kernel<<<sec_cdiv(n, 256), 256, 0, s->st>>>(s->core->incU, s->d_perm.as<int>(), s->nu, s->bu,
                                                                   s->inc_user.as<double>());
      NL_CUDA(cudaGetLastError());
      NL_CUDA(cudaMemcpyAsync(incU, s->inc_user.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s->st));
    }
    if (incV && s->nv > 0)
      NL_CUDA(cudaMemcpyAsync(incV, s->core->incV, sizeof(double) * 3 * s->nv, cudaMemcpyDeviceToHost, s->st));
    NL_CUDA(cudaStreamSynchronize(s->st));
    if (ok) *ok = good ? 1 : 0;
  } catch (const HostError& e) {
    return e.s;
  }
  return NL_OK;
}

nl_status nl_section_lm_solve(nl_section* s, const nl_lm_settings* st, nl_solve_report* rep, double* trace,
                              int trace_cap) {
  if (!s || !st) return NL_ERR_ARG;
  if (!s->ready || !s->have_cb || !s->cb.backup || !s->cb.rollback) return NL_ERR_STATE;
  try {
    NL_CUDA(cudaSetDevice(s->device));
    SectionOps P{s};
    int ntr = 0, its = 0, subs = 0;
    double mu = 0.0;
    cudaEvent_t e0, e1;
    NL_CUDA(cudaEventCreate(&e0));
    NL_CUDA(cudaEventCreate(&e1));
    NL_CUDA(cudaEventRecord(e0, s->st));
    const int reason = host_lm_loop(P, *st, trace, std::max(0, trace_cap), &ntr, &its, &subs, &mu);
    NL_CUDA(cudaEventRecord(e1, s->st));
    NL_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rep) {
      rep->reason = reason;
      rep->iterations = its;
      rep->subiterations = subs;
      rep->n_trace = ntr;
      rep->chi2 = s->chi2;
      rep->mu = mu;
      rep->device_ms = ms;
    }
  } catch (const HostError& e) {
    return e.s;
  }
  return NL_OK;
}

nl_status nl_section_gn_solve(nl_section* s, const nl_gn_settings* st, nl_solve_report* rep, double* trace,
                              int trace_cap) {
  if (!s || !st) return NL_ERR_ARG;
  if (!s->ready || !s->have_cb) return NL_ERR_STATE;
  try {
    NL_CUDA(cudaSetDevice(s->device));
    SectionOps P{s};
    int ntr = 0, its = 0;
    cudaEvent_t e0, e1;
    NL_CUDA(cudaEventCreate(&e0));
    NL_CUDA(cudaEventCreate(&e1));
    NL_CUDA(cudaEventRecord(e0, s->st));
    const int reason = host_gn_loop(P, *st, trace, std::max(0, trace_cap), &ntr, &its);
    NL_CUDA(cudaEventRecord(e1, s->st));
    NL_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rep) {
      rep->reason = reason;
      rep->iterations = its;
      rep->subiterations = its;
      rep->n_trace = ntr;
      rep->chi2 = s->chi2;
      rep->mu = 0.0;
      rep->device_ms = ms;
    }
  } catch (const HostError& e) {
    return e.s;
  }
  return NL_OK;
}

}  // extern "C"
