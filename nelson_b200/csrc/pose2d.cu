// pose2d.cu -- a SingleSection on the device: SE(2) poses aligned by
// point-to-line edges between 2D scans.
//
// The reference's single-section problem (nelson/SingleSection.hpp:63-139,
// solved by nelson/LevenbergMarquardt.hpp:36-146 and nelson/GaussNewton.hpp:
// 32-127 with SolverCholeskyDense, nelson/SolverCholeskyDense.hpp:39-67) as
// its tests build it (nelson/tests/testGaussNewton2DScansAlign.cpp:36-120):
// every edge joins a model pose a and a target pose b and holds K model
// points m_k with normals n_k (in a's frame) and K target points q_k (in b's
// frame).  With X_m = T_a m, N = R_a n, X_t = T_b q the residual is
// e_k = (X_m - X_t) . N, the cost sum_k e_k^2, and under the left perturbation
// T <- exp(d) T, d = (v_x, v_y, w), the Jacobians are g and -g with
// g = (N_x, N_y, X_t,x N_y - X_t,y N_x).  So an edge contributes Hs = sum g g'
// and bs = sum g e:  U_aa += Hs, U_bb += Hs, U_ab -= Hs, b_a += bs, b_b -= bs.
//
// Device layout: poses (x, y, theta) per slot (variable poses first, fixed
// after), the edges' point triples in edge order.  pose2d_edge_kernel: one
// CTA per edge, the K points strided over the threads, per-thread partials
// reduced in a fixed order into the edge's (chi2, Hs, bs).  pose2d_assemble:
// one thread per entry of a U block / of b, summing its edges' contributions
// in edge order (lists built at structureReady), so the Hessian is
// bit-reproducible.  The reduced system is U itself (no V / W blocks), solved
// by the library's tiled Cholesky (SchurCore with nv = 0: damping diag (1 +
// rel) + abs, then factor and solve), dense or envelope.  oplus applies the
// SE(2) exponential on the left: theta += w, t <- R(w) t + V(w) v with
// V(w) = [[sin w / w, -(1 - cos w) / w], [(1 - cos w) / w, sin w / w]].
// The LM / GN control runs on the host (host_lm.cuh), one device round trip
// per step.
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

inline int p2_cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }
constexpr int kEdgeVals = 10;  // chi2, Hs (00 01 02 11 12 22), bs (0 1 2)

__device__ __forceinline__ double p2_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One warp per chunk of at most kChunkPts points of one edge (8 warps per
// CTA): the lane-strided points, 16-byte (x, y) loads, the 10 values
// butterfly-reduced over the warp, lane i writing value i of the chunk's
// record.  A fixed order everywhere, so the records are bit-reproducible.
constexpr int kChunkPts = 128;
constexpr int kChunkWarps = 8;
static __global__ void __launch_bounds__(32 * kChunkWarps, 4) pose2d_edge_kernel(
    const double* __restrict__ pose, const int* __restrict__ ea, const int* __restrict__ eb,
    const int* __restrict__ chunk_edge, const int* __restrict__ chunk_p0, int nchunks,
    const int* __restrict__ pt_ptr, const double2* __restrict__ mp, const double2* __restrict__ mn,
    const double2* __restrict__ tp, double* __restrict__ out, int with_h) {
  const int c = blockIdx.x * kChunkWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (c >= nchunks) return;  // the whole warp
  const int e = chunk_edge[c];
  const int k0 = chunk_p0[c], k1 = min(k0 + kChunkPts, pt_ptr[e + 1]);
  const double* A = pose + 3 * (size_t)ea[e];
  const double* B = pose + 3 * (size_t)eb[e];
  double ca, sa, cb, sb;
  sincos(A[2], &sa, &ca);
  sincos(B[2], &sb, &cb);
  const double ax = A[0], ay = A[1], bx = B[0], by = B[1];
  double v[kEdgeVals];
#pragma unroll
  for (int i = 0; i < kEdgeVals; i++) v[i] = 0.0;
#pragma unroll 4
  for (int k = k0 + lane; k < k1; k += 32) {
    const double2 m = mp[k], n = mn[k], q = tp[k];
    const double xm0 = ca * m.x - sa * m.y + ax, xm1 = sa * m.x + ca * m.y + ay;
    const double N0 = ca * n.x - sa * n.y, N1 = sa * n.x + ca * n.y;
    const double xt0 = cb * q.x - sb * q.y + bx, xt1 = sb * q.x + cb * q.y + by;
    const double err = (xm0 - xt0) * N0 + (xm1 - xt1) * N1;
    v[0] += err * err;
    if (with_h) {
      const double g0 = N0, g1 = N1, g2 = xt0 * N1 - xt1 * N0;
      v[1] += g0 * g0;
      v[2] += g0 * g1;
      v[3] += g0 * g2;
      v[4] += g1 * g1;
      v[5] += g1 * g2;
      v[6] += g2 * g2;
      v[7] += g0 * err;
      v[8] += g1 * err;
      v[9] += g2 * err;
    }
  }
  double mine = 0.0;
#pragma unroll
  for (int i = 0; i < kEdgeVals; i++) {
    const double t = p2_warp_sum(v[i]);
    if (lane == i) mine = t;
  }
  if (lane < kEdgeVals) out[(size_t)c * kEdgeVals + lane] = mine;
}

// an edge's record: its chunks' records summed in chunk order; the edge's
// cost also goes to the contiguous echi (read by the chi2 reduction)
static __global__ void pose2d_chunk_sum_kernel(const double* __restrict__ cv, const int* __restrict__ cptr, int ne,
                                               double* __restrict__ ev, double* __restrict__ echi) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ne * kEdgeVals) return;
  const int e = t / kEdgeVals, i = t - e * kEdgeVals;
  double s = 0.0;
  for (int c = cptr[e]; c < cptr[e + 1]; c++) s += cv[(size_t)c * kEdgeVals + i];
  ev[t] = s;
  if (i == 0) echi[e] = s;
}

// U block entries and b entries from the edges: item q of the (uid, entry)
// and (internal pose, component) lists; each sums its (edge, sign) list in
// order.  Hs entry (r, c) -> index in the edge record.
__device__ __forceinline__ int hs_index(int r, int c) {
  const int i = min(r, c), j = max(r, c);
  return 1 + (i == 0 ? j : (i == 1 ? 2 + j : 5));
}

template <typename T>
static __global__ void pose2d_assemble_kernel(const double* __restrict__ ev, int nU, int LU,
                                              const int* __restrict__ u_ptr, const int* __restrict__ u_edge,
                                              const signed char* __restrict__ u_sign, int nb,
                                              const int* __restrict__ b_ptr, const int* __restrict__ b_edge,
                                              const signed char* __restrict__ b_sign, T* __restrict__ U,
                                              T* __restrict__ bU) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < 9 * nU) {
    const int uid = t / 9, ent = t - 9 * uid, r = ent / 3, c = ent - 3 * r;
    const int hi = hs_index(r, c);
    double s = 0.0;
    for (int q = u_ptr[uid]; q < u_ptr[uid + 1]; q++) s += u_sign[q] * ev[(size_t)u_edge[q] * kEdgeVals + hi];
    U[(size_t)uid * LU + ent] = (T)s;
  } else if (t < 9 * nU + 3 * nb) {
    const int q0 = t - 9 * nU, i = q0 / 3, k = q0 - 3 * i;
    double s = 0.0;
    for (int q = b_ptr[i]; q < b_ptr[i + 1]; q++) s += b_sign[q] * ev[(size_t)b_edge[q] * kEdgeVals + 7 + k];
    bU[3 * (size_t)i + k] = (T)s;
  }
}

// chi2 = sum of the edges' costs (contiguous), in a fixed order
static __global__ void pose2d_chi2_kernel(const double* __restrict__ echi, int ne, double* __restrict__ out) {
  __shared__ double red[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double s = 0.0;
#pragma unroll 4
  for (int e = tid; e < ne; e += blockDim.x) s += echi[e];
  s = p2_warp_sum(s);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    *out = t;
  }
}

// T_u <- exp(d) T_u for the variable poses, d at the internal position perm[u]
static __global__ void pose2d_oplus_kernel(double* __restrict__ pose, const int* __restrict__ perm, int nv,
                                           const double* __restrict__ inc) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nv) return;
  const double* d = inc + 3 * (size_t)perm[u];
  const double vx = d[0], vy = d[1], w = d[2];
  double sw, cw;
  sincos(w, &sw, &cw);
  double a, b;  // V(w) = [[a, -b], [b, a]]
  if (fabs(w) > 1e-9) {
    a = sw / w;
    b = (1.0 - cw) / w;
  } else {
    a = 1.0 - w * w / 6.0;
    b = 0.5 * w;
  }
  double* p = pose + 3 * (size_t)u;
  const double x = p[0], y = p[1];
  p[0] = cw * x - sw * y + (a * vx - b * vy);
  p[1] = sw * x + cw * y + (b * vx + a * vy);
  p[2] = p[2] + w;
}

}  // namespace
}  // namespace nl

using namespace nl;

struct nl_pose2d {
  int nv = 0, nf = 0, device = 0, precision = NL_PREC_FP64;
  bool ready = false;
  cudaStream_t st = nullptr;
  cublasHandle_t cublas = nullptr;
  DevBuf ws, pose, pose_bck, ebuf, scal, lam;
  DevBuf d_ea, d_eb, d_ptr, d_mp, d_mn, d_tp, d_perm, d_uptr, d_uedge, d_usign, d_bptr, d_bedge, d_bsign;
  DevBuf d_cedge, d_cp0, d_cptr, cbuf;  // point chunks of the edges (kChunkPts each)
  DevBuf echi;                          // per-edge cost, contiguous
  int nchunks = 0;
  std::unique_ptr<SchurCore> core;
  std::vector<int> ea, eb, pt_ptr{0}, perm;
  std::vector<std::pair<int, int>> blocks;  // U pattern, (col, row) internal, CSC order
  std::vector<double> mp, mn, tp, pose_h;
  int nU = 0;
  double chi2 = 0.0;
  double* pin = nullptr;
  std::vector<double> bU_h;  // b of the last update(true), internal order
  ~nl_pose2d() {
    core.reset();
    if (cublas) cublasDestroy(cublas);
    if (pin) cudaFreeHost(pin);
    if (st) cudaStreamDestroy(st);
  }
};

namespace {

#define P2_CUDA(x)                                       \
  do {                                                   \
    if ((x) != cudaSuccess) throw HostError{NL_ERR_CUDA}; \
  } while (0)

// The problem operations the LM / GN loops need (the problem concept of
// nelson/LevenbergMarquardt.hpp:41-136, with the solver's increment).
struct Pose2DOps {
  nl_pose2d* h;
  void update(bool hess) {
    const int ne = (int)h->ea.size();
    if (ne > 0) {
      pose2d_edge_kernel<<<p2_cdiv(h->nchunks, kChunkWarps), 32 * kChunkWarps, 0, h->st>>>(
          h->pose.as<double>(), h->d_ea.as<int>(), h->d_eb.as<int>(), h->d_cedge.as<int>(), h->d_cp0.as<int>(),
          h->nchunks, h->d_ptr.as<int>(), h->d_mp.as<double2>(), h->d_mn.as<double2>(), h->d_tp.as<double2>(),
          h->cbuf.as<double>(), hess ? 1 : 0);
      pose2d_chunk_sum_kernel<<<p2_cdiv(ne * kEdgeVals, 256), 256, 0, h->st>>>(h->cbuf.as<double>(),
                                                                               h->d_cptr.as<int>(), ne,
                                                                               h->ebuf.as<double>(),
                                                                               h->echi.as<double>());
      P2_CUDA(cudaGetLastError());
    }
    if (hess) {
      const int n = 9 * h->nU + 3 * h->nv;
      const int LU = h->precision == NL_PREC_FP64 ? Layout<double, 3>::U : Layout<float, 3>::U;
      if (n > 0) {
        if (h->precision == NL_PREC_FP64)
          pose2d_assemble_kernel<double><<<p2_cdiv(n, 128), 128, 0, h->st>>>(
              h->ebuf.as<double>(), h->nU, LU, h->d_uptr.as<int>(), h->d_uedge.as<int>(),
              h->d_usign.as<signed char>(), h->nv, h->d_bptr.as<int>(), h->d_bedge.as<int>(),
              h->d_bsign.as<signed char>(), (double*)h->core->dU(), (double*)h->core->dbU());
        else
          pose2d_assemble_kernel<float><<<p2_cdiv(n, 128), 128, 0, h->st>>>(
              h->ebuf.as<double>(), h->nU, LU, h->d_uptr.as<int>(), h->d_uedge.as<int>(),
              h->d_usign.as<signed char>(), h->nv, h->d_bptr.as<int>(), h->d_bedge.as<int>(),
              h->d_bsign.as<signed char>(), (float*)h->core->dU(), (float*)h->core->dbU());
        P2_CUDA(cudaGetLastError());
      }
    }
    pose2d_chi2_kernel<<<1, 1024, 0, h->st>>>(h->echi.as<double>(), ne, h->scal.as<double>());
    P2_CUDA(cudaGetLastError());
    P2_CUDA(cudaMemcpyAsync(h->pin, h->scal.p, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    if (hess) read_b();
    P2_CUDA(cudaStreamSynchronize(h->st));
    h->chi2 = h->pin[0];
  }
  void read_b() {
    const int n = 3 * h->nv;
    h->bU_h.assign(n, 0.0);
    if (n == 0) return;
    if (h->precision == NL_PREC_FP64) {
      P2_CUDA(cudaMemcpyAsync(h->bU_h.data(), h->core->dbU(), sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
    } else {
      std::vector<float> f(n);
      P2_CUDA(cudaMemcpyAsync(f.data(), h->core->dbU(), sizeof(float) * n, cudaMemcpyDeviceToHost, h->st));
      P2_CUDA(cudaStreamSynchronize(h->st));
      for (int i = 0; i < n; i++) h->bU_h[i] = f[i];
    }
  }
  double chi2() const { return h->chi2; }
  double max_abs_b() const {
    double m = 0.0;
    for (double x : h->bU_h) m = std::max(m, std::fabs(x));
    return m;
  }
  double max_abs_hdiag() {
    double* dv = h->scal.as<double>() + 1;
    host_check(h->core->enqueue_hdiag(dv));
    P2_CUDA(cudaMemcpyAsync(h->pin + 1, dv, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    P2_CUDA(cudaStreamSynchronize(h->st));
    return h->pin[1];
  }
  std::vector<double> inc;
  bool compute_increment(double rel, double abs_) {
    h->pin[2] = rel;
    h->pin[3] = abs_;
    P2_CUDA(cudaMemcpyAsync(h->lam.p, h->pin + 2, 2 * sizeof(double), cudaMemcpyHostToDevice, h->st));
    int* status = reinterpret_cast<int*>(h->lam.as<double>() + 2);
    P2_CUDA(cudaMemsetAsync(status, 0, sizeof(int), h->st));
    host_check(h->core->enqueue_increment(h->lam.as<double>(), status, nullptr));
    const int n = 3 * h->nv;
    inc.assign(n, 0.0);
    if (n) P2_CUDA(cudaMemcpyAsync(inc.data(), h->core->incU, sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
    P2_CUDA(cudaMemcpyAsync(h->pin + 4, status, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    P2_CUDA(cudaStreamSynchronize(h->st));
    int stt = 0;
    memcpy(&stt, h->pin + 4, sizeof(int));
    if (stt & ST_SPIN_TIMEOUT) throw HostError{NL_ERR_TIMEOUT};
    return stt == 0;
  }
  double inc_sqnorm() const {
    double s = 0.0;
    for (double x : inc) s += x * x;
    return s;
  }
  // computeRhoChi2Change (nelson/SingleSection.h:206-213) with the chi2 of
  // the candidate already evaluated
  double rho(double mu, double oldChi2) const {
    double den = 0.0;
    for (size_t i = 0; i < inc.size(); i++) den += inc[i] * (mu * inc[i] - h->bU_h[i]);
    return (oldChi2 - h->chi2) / den;
  }
  void oplus() {
    if (h->nv > 0) {
      pose2d_oplus_kernel<<<p2_cdiv(h->nv, 128), 128, 0, h->st>>>(h->pose.as<double>(), h->d_perm.as<int>(), h->nv,
                                                               h->core->incU);
      P2_CUDA(cudaGetLastError());
    }
  }
  void backup() {
    P2_CUDA(cudaMemcpyAsync(h->pose_bck.p, h->pose.p, h->pose.bytes, cudaMemcpyDeviceToDevice, h->st));
  }
  void rollback() {
    P2_CUDA(cudaMemcpyAsync(h->pose.p, h->pose_bck.p, h->pose.bytes, cudaMemcpyDeviceToDevice, h->st));
  }
};

}  // namespace

extern "C" {

nl_status nl_pose2d_create(int nv, int nf, int precision, int device, nl_pose2d** out) {
  if (nv < 1 || nf < 0 || !out || (precision != NL_PREC_FP64 && precision != NL_PREC_MIXED)) return NL_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<nl_pose2d> h(new nl_pose2d());
  h->nv = nv;
  h->nf = nf;
  h->precision = precision;
  h->device = device;
  h->perm.resize(nv);
  for (int i = 0; i < nv; i++) h->perm[i] = i;
  h->pose_h.assign(3 * (size_t)(nv + nf), 0.0);
  NL_CUDA(cudaSetDevice(device));
  NL_CUDA(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  NL_CUDA(cudaMallocHost(&h->pin, 64));
  *out = h.release();
  return NL_OK;
}

nl_status nl_pose2d_destroy(nl_pose2d* h) {
  if (!h) return NL_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->st) cudaStreamSynchronize(h->st);
  delete h;
  return NL_OK;
}

nl_status nl_pose2d_set_poses(nl_pose2d* h, const double* var_xyt, const double* fix_xyt) {
  if (!h) return NL_ERR_ARG;
  if (var_xyt) std::copy(var_xyt, var_xyt + 3 * (size_t)h->nv, h->pose_h.begin());
  if (fix_xyt) std::copy(fix_xyt, fix_xyt + 3 * (size_t)h->nf, h->pose_h.begin() + 3 * (size_t)h->nv);
  if (h->ready) {
    NL_CUDA(cudaSetDevice(h->device));
    NL_CUDA(cudaMemcpyAsync(h->pose.p, h->pose_h.data(), sizeof(double) * h->pose_h.size(), cudaMemcpyHostToDevice,
                            h->st));
    NL_CUDA(cudaStreamSynchronize(h->st));
  }
  return NL_OK;
}

nl_status nl_pose2d_get_poses(nl_pose2d* h, double* var_xyt) {
  if (!h || !var_xyt) return NL_ERR_ARG;
  if (!h->ready) {
    std::copy(h->pose_h.begin(), h->pose_h.begin() + 3 * (size_t)h->nv, var_xyt);
    return NL_OK;
  }
  NL_CUDA(cudaSetDevice(h->device));
  if (h->nv) NL_CUDA(cudaMemcpyAsync(var_xyt, h->pose.p, sizeof(double) * 3 * h->nv, cudaMemcpyDeviceToHost, h->st));
  NL_CUDA(cudaStreamSynchronize(h->st));
  return NL_OK;
}

nl_status nl_pose2d_add_edge(nl_pose2d* h, int a, int a_fixed, int b, int b_fixed, int npts,
                             const double* model_pts, const double* model_normals, const double* target_pts) {
  if (!h || h->ready || npts < 0 || (npts > 0 && (!model_pts || !model_normals || !target_pts))) return NL_ERR_ARG;
  const int sa = a_fixed ? h->nv + a : a, sb = b_fixed ? h->nv + b : b;
  if (a < 0 || b < 0 || (a_fixed ? a >= h->nf : a >= h->nv) || (b_fixed ? b >= h->nf : b >= h->nv)) return NL_ERR_ARG;
  if (sa == sb || (a_fixed && b_fixed)) return NL_ERR_ARG;
  h->ea.push_back(sa);
  h->eb.push_back(sb);
  h->mp.insert(h->mp.end(), model_pts, model_pts + 2 * (size_t)npts);
  h->mn.insert(h->mn.end(), model_normals, model_normals + 2 * (size_t)npts);
  h->tp.insert(h->tp.end(), target_pts, target_pts + 2 * (size_t)npts);
  h->pt_ptr.push_back(h->pt_ptr.back() + npts);
  return NL_OK;
}

nl_status nl_pose2d_set_user2internal(nl_pose2d* h, const int* perm) {
  if (!h || !perm || h->ready) return NL_ERR_ARG;
  std::vector<char> seen(h->nv, 0);
  for (int i = 0; i < h->nv; i++) {
    if (perm[i] < 0 || perm[i] >= h->nv || seen[perm[i]]) return NL_ERR_ARG;
    seen[perm[i]] = 1;
  }
  std::copy(perm, perm + h->nv, h->perm.begin());
  return NL_OK;
}

// SingleSection::permuteAMD (nelson/SingleSection.hpp:33-52): the approximate
// minimum degree order of the pose graph (variable poses joined by an edge)
nl_status nl_pose2d_permute_amd(nl_pose2d* h) {
  if (!h || h->ready) return NL_ERR_ARG;
  std::vector<int> r, c;
  for (size_t e = 0; e < h->ea.size(); e++)
    if (h->ea[e] < h->nv && h->eb[e] < h->nv) {
      r.push_back(h->ea[e]);
      c.push_back(h->eb[e]);
    }
  return nl_amd_order(h->nv, (int)r.size(), r.data(), c.data(), h->perm.data());
}

// Reverse Cuthill-McKee order of the same pose graph: the order that keeps
// U's profile narrow for the envelope solver (on a chain with short loop
// closures the band stays within a tile or two, where the fill-reducing
// minimum degree order scatters it).  Each edge between two variable poses
// enters as a two-pose clique.
nl_status nl_pose2d_permute_rcm(nl_pose2d* h) {
  if (!h || h->ready) return NL_ERR_ARG;
  std::vector<int> cam, pt;
  int k = 0;
  for (size_t e = 0; e < h->ea.size(); e++)
    if (h->ea[e] < h->nv && h->eb[e] < h->nv) {
      cam.push_back(h->ea[e]);
      cam.push_back(h->eb[e]);
      pt.push_back(k);
      pt.push_back(k);
      k++;
    }
  return nl_rcm_order(h->nv, k, (int)cam.size(), cam.data(), pt.data(), h->perm.data());
}

// SingleSection::structureReady: the U pattern (upper CSC in internal order),
// the (edge, sign) lists of every U block and b entry, device buffers, the
// tiled Cholesky of the reduced system U.
nl_status nl_pose2d_structure_ready(nl_pose2d* h) {
  if (!h || h->ready) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(h->device));
  const int nv = h->nv, ne = (int)h->ea.size();
  // U blocks: (i, i) for every variable pose, (i, j) i < j for pose pairs with an edge
  std::vector<std::pair<int, int>>& blocks = h->blocks;  // (col, row), sorted = CSC order
  blocks.clear();
  for (int i = 0; i < nv; i++) blocks.push_back({i, i});
  for (int e = 0; e < ne; e++)
    if (h->ea[e] < nv && h->eb[e] < nv) {
      const int i = h->perm[h->ea[e]], j = h->perm[h->eb[e]];
      blocks.push_back({std::max(i, j), std::min(i, j)});
    }
  std::sort(blocks.begin(), blocks.end());
  blocks.erase(std::unique(blocks.begin(), blocks.end()), blocks.end());
  h->nU = (int)blocks.size();
  auto uid_of = [&](int r, int c) {
    const auto it = std::lower_bound(blocks.begin(), blocks.end(), std::make_pair(c, r));
    return (int)(it - blocks.begin());
  };
  std::vector<std::vector<std::pair<int, int>>> ul(h->nU), bl(nv);
  for (int e = 0; e < ne; e++) {
    const bool va = h->ea[e] < nv, vb = h->eb[e] < nv;
    const int ia = va ? h->perm[h->ea[e]] : -1, ib = vb ? h->perm[h->eb[e]] : -1;
    if (va) {
      ul[uid_of(ia, ia)].push_back({e, 1});
      bl[ia].push_back({e, 1});
    }
    if (vb) {
      ul[uid_of(ib, ib)].push_back({e, 1});
      bl[ib].push_back({e, -1});
    }
    if (va && vb) ul[uid_of(std::min(ia, ib), std::max(ia, ib))].push_back({e, -1});
  }
  std::vector<int> uptr{0}, uedge, bptr{0}, bedge;
  std::vector<signed char> usign, bsign;
  for (auto& l : ul) {
    for (auto& x : l) {
      uedge.push_back(x.first);
      usign.push_back((signed char)x.second);
    }
    uptr.push_back((int)uedge.size());
  }
  for (auto& l : bl) {
    for (auto& x : l) {
      bedge.push_back(x.first);
      bsign.push_back((signed char)x.second);
    }
    bptr.push_back((int)bedge.size());
  }
  nl_status s;
  if ((s = upload(h->d_ea, h->ea, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_eb, h->eb, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_ptr, h->pt_ptr, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_mp, h->mp, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_mn, h->mn, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_tp, h->tp, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_perm, h->perm, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_uptr, uptr, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_uedge, uedge, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_usign, usign, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_bptr, bptr, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_bedge, bedge, h->st)) != NL_OK) return s;
  if ((s = upload(h->d_bsign, bsign, h->st)) != NL_OK) return s;
  if ((s = upload(h->pose, h->pose_h, h->st)) != NL_OK) return s;
  if ((s = h->pose_bck.alloc(h->pose.bytes)) != NL_OK) return s;
  if ((s = h->ebuf.alloc(sizeof(double) * kEdgeVals * (size_t)std::max(ne, 1))) != NL_OK) return s;
  {
    // point chunks: every edge gets ceil(npts / kChunkPts) of them, at least one
    std::vector<int> cedge, cp0, cptr{0};
    for (int e = 0; e < ne; e++) {
      const int p0 = h->pt_ptr[e], p1 = h->pt_ptr[e + 1];
      int p = p0;
      do {
        cedge.push_back(e);
        cp0.push_back(p);
        p += kChunkPts;
      } while (p < p1);
      cptr.push_back((int)cedge.size());
    }
    h->nchunks = (int)cedge.size();
    if ((s = upload(h->d_cedge, cedge, h->st)) != NL_OK) return s;
    if ((s = upload(h->d_cp0, cp0, h->st)) != NL_OK) return s;
    if ((s = upload(h->d_cptr, cptr, h->st)) != NL_OK) return s;
    if ((s = h->cbuf.alloc(sizeof(double) * kEdgeVals * (size_t)std::max(h->nchunks, 1))) != NL_OK) return s;
    if ((s = h->echi.alloc(sizeof(double) * (size_t)std::max(ne, 1))) != NL_OK) return s;
  }
  if ((s = h->scal.alloc(64)) != NL_OK) return s;
  if ((s = h->lam.alloc(64)) != NL_OK) return s;
  // the reduced system: U only (bu = 3, nv = 0)
  if (h->precision == NL_PREC_FP64) {
    if (cublasCreate(&h->cublas) != CUBLAS_STATUS_SUCCESS) return NL_ERR_CUDA;
    cublasSetStream(h->cublas, h->st);
    if ((s = h->ws.alloc(64u << 20)) != NL_OK) return s;
    cublasSetWorkspace(h->cublas, h->ws.p, h->ws.bytes);
  }
  h->core = make_schur_core(h->precision, 3, h->cublas);
  if (!h->core) return NL_ERR_UNSUPPORTED;
  h->core->refine_sweeps = h->precision == NL_PREC_MIXED ? 1 : 0;
  h->core->keep_schur = 0;
  h->core->use_tc = h->precision == NL_PREC_MIXED ? 1 : 0;
  SchurStructure ss;
  ss.bc = 3;
  ss.nci = nv;
  ss.np = 0;
  for (auto& b : blocks) {
    ss.u_r.push_back(b.second);
    ss.u_c.push_back(b.first);
  }
  if ((s = h->core->setup(ss, h->st)) != NL_OK) return s;
  NL_CUDA(cudaStreamSynchronize(h->st));
  h->ready = true;
  return NL_OK;
}

// The Hessian of the last update(true) as a dense symmetric 3 nv x 3 nv
// matrix and b, both in user pose order (SingleSection::hessian().H / b)
nl_status nl_pose2d_get_hessian(nl_pose2d* h, double* H, double* b) {
  if (!h) return NL_ERR_ARG;
  if (!h->ready) return NL_ERR_STATE;
  NL_CUDA(cudaSetDevice(h->device));
  const size_t n = 3 * (size_t)h->nv;
  const bool f64 = h->precision == NL_PREC_FP64;
  const int LU = f64 ? Layout<double, 3>::U : Layout<float, 3>::U;
  std::vector<double> U((size_t)h->nU * LU), bu(n);
  if (f64) {
    if (h->nU)
      NL_CUDA(cudaMemcpyAsync(U.data(), h->core->dU(), sizeof(double) * U.size(), cudaMemcpyDeviceToHost, h->st));
    if (n) NL_CUDA(cudaMemcpyAsync(bu.data(), h->core->dbU(), sizeof(double) * n, cudaMemcpyDeviceToHost, h->st));
    NL_CUDA(cudaStreamSynchronize(h->st));
  } else {
    std::vector<float> Uf(U.size()), bf(n);
    if (h->nU)
      NL_CUDA(cudaMemcpyAsync(Uf.data(), h->core->dU(), sizeof(float) * Uf.size(), cudaMemcpyDeviceToHost, h->st));
    if (n) NL_CUDA(cudaMemcpyAsync(bf.data(), h->core->dbU(), sizeof(float) * n, cudaMemcpyDeviceToHost, h->st));
    NL_CUDA(cudaStreamSynchronize(h->st));
    std::copy(Uf.begin(), Uf.end(), U.begin());
    std::copy(bf.begin(), bf.end(), bu.begin());
  }
  std::vector<int> user(h->nv);
  for (int u = 0; u < h->nv; u++) user[h->perm[u]] = u;
  if (H) {
    std::fill(H, H + n * n, 0.0);
    for (int q = 0; q < h->nU; q++) {
      const int r = user[h->blocks[q].second], c = user[h->blocks[q].first];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          const double v = U[(size_t)q * LU + 3 * i + j];
          H[(3 * (size_t)r + i) * n + 3 * (size_t)c + j] = v;
          H[(3 * (size_t)c + j) * n + 3 * (size_t)r + i] = v;
        }
    }
  }
  if (b)
    for (int u = 0; u < h->nv; u++)
      for (int k = 0; k < 3; k++) b[3 * (size_t)u + k] = bu[3 * (size_t)h->perm[u] + k];
  return NL_OK;
}

nl_status nl_pose2d_set_solver_kind(nl_pose2d* h, int kind) {
  if (!h || !h->ready) return NL_ERR_STATE;
  if (kind != NL_SOLVER_DENSE && kind != NL_SOLVER_ENVELOPE) return NL_ERR_ARG;
  h->core->envelope = kind == NL_SOLVER_ENVELOPE ? 1 : 0;
  return NL_OK;
}

nl_status nl_pose2d_update(nl_pose2d* h, int hessian, double* chi2) {
  if (!h) return NL_ERR_ARG;
  if (!h->ready) return NL_ERR_STATE;
  try {
    NL_CUDA(cudaSetDevice(h->device));
    Pose2DOps P{h};
    P.update(hessian != 0);
    if (chi2) *chi2 = h->chi2;
  } catch (const HostError& e) {
    return e.s;
  }
  return NL_OK;
}

nl_status nl_pose2d_lm_solve(nl_pose2d* h, const nl_lm_settings* st, nl_solve_report* rep, double* trace,
                             int trace_cap) {
  if (!h || !st) return NL_ERR_ARG;
  if (!h->ready) return NL_ERR_STATE;
  try {
    NL_CUDA(cudaSetDevice(h->device));
    Pose2DOps P{h};
    int ntr = 0, its = 0, subs = 0;
    cudaEvent_t e0, e1;
    NL_CUDA(cudaEventCreate(&e0));
    NL_CUDA(cudaEventCreate(&e1));
    NL_CUDA(cudaEventRecord(e0, h->st));
    const int reason = host_lm_loop(P, *st, trace, std::max(0, trace_cap), &ntr, &its, &subs, nullptr);
    NL_CUDA(cudaEventRecord(e1, h->st));
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
      rep->chi2 = h->chi2;
      rep->mu = 0.0;
      rep->device_ms = ms;
    }
  } catch (const HostError& e) {
    return e.s;
  }
  return NL_OK;
}

nl_status nl_pose2d_gn_solve(nl_pose2d* h, const nl_gn_settings* st, nl_solve_report* rep, double* trace,
                             int trace_cap) {
  if (!h || !st) return NL_ERR_ARG;
  if (!h->ready) return NL_ERR_STATE;
  try {
    NL_CUDA(cudaSetDevice(h->device));
    Pose2DOps P{h};
    int ntr = 0, its = 0;
    cudaEvent_t e0, e1;
    NL_CUDA(cudaEventCreate(&e0));
    NL_CUDA(cudaEventCreate(&e1));
    NL_CUDA(cudaEventRecord(e0, h->st));
    const int reason = host_gn_loop(P, *st, trace, std::max(0, trace_cap), &ntr, &its);
    NL_CUDA(cudaEventRecord(e1, h->st));
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
      rep->chi2 = h->chi2;
      rep->mu = 0.0;
      rep->device_ms = ms;
    }
  } catch (const HostError& e) {
    return e.s;
  }
  return NL_OK;
}

}  // extern "C"
