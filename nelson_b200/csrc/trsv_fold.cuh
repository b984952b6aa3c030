// trsv_fold.cuh -- triangular solves with the factor of S, tile row by tile
// row, with two changes to the look-back of cholesky.cuh's trsv kernels that
// shorten the chain from one tile to the next:
//   * a solution value is its own readiness marker: the solution vector is
//     filled with an "unsolved" NaN pattern (a payload no arithmetic
//     produces) before the sweep, and a consumer polls the values it needs
//     until none is unsolved, so there is no separate flag, no CTA barrier
//     and no release fence between a tile's values and its consumers; each
//     warp publishes its own 8 rows as soon as they are ready;
//   * the last off-diagonal tile of a row is folded into the diagonal
//     inverse: forward, y_I = c_I - M_I y_{I-1} with M_I = inv(L_II) L_I,I-1
//     and c_I = inv(L_II) (b_I - sum_{J < I-1} L_IJ y_J), so after y_{I-1}
//     arrives one 128 x 128 product (from registers) and a warp reduction
//     remain; backward, x_I = d_I - P_I x_{I+1} with P_I = inv(L_II)'
//     L_I+1,I' (stored row-major in that product's orientation) and
//     d_I = inv(L_II)' (y_I - sum_{J > I+1} L_JI' x_J).
// M_I and P_I are formed once per factorisation (fold_kernel).  CTAs take
// tiles in ticket order, so a CTA only waits for tiles held by CTAs that
// started before it; every wait is bounded, and a CTA that gives up records
// ST_SPIN_TIMEOUT and publishes nothing, so its consumers give up in turn.
#pragma once

#include "cholesky.cuh"

namespace nl {

constexpr long long kUnsolvedBits = 0x7FF40000DEAD5AB1ll;

__device__ __forceinline__ double unsolved_value() { return __longlong_as_double(kUnsolvedBits); }
__device__ __forceinline__ bool is_unsolved(double v) { return __double_as_longlong(v) == kUnsolvedBits; }

__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];\n" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_f64(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;\n" ::"l"(p), "d"(v) : "memory");
}

// Poll 4 consecutive values until none is unsolved; false after `limit` polls.
__device__ inline bool wait_values4(const double* p, double* v, long long limit) {
  for (long long it = 0;; it++) {
    v[0] = ld_relaxed_f64(p);
    v[1] = ld_relaxed_f64(p + 1);
    v[2] = ld_relaxed_f64(p + 2);
    v[3] = ld_relaxed_f64(p + 3);
    if (!is_unsolved(v[0]) && !is_unsolved(v[1]) && !is_unsolved(v[2]) && !is_unsolved(v[3])) return true;
    if (it >= limit) return false;
    if (it > 4096) __nanosleep(64);
  }
}

__device__ __forceinline__ double warp_all_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Both solution vectors unsolved, both tickets zero.
static __global__ void unsolved_fill_kernel(double* __restrict__ y, double* __restrict__ x, int n,
                                            int* __restrict__ tickets, const int* __restrict__ active) {
  if (active && !*active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    y[i] = unsolved_value();
    x[i] = unsolved_value();
  }
  if (i < 2) tickets[i] = 0;
}

// M_I = inv(L_II) L_I,I-1 (I = 1 .. ntiles - 1) and P_I = inv(L_II)' L_I+1,I'
// (I = 0 .. ntiles - 2), 128 x 128 x 128 products, one CTA each: 256 threads,
// 8 x 8 outputs per thread, 32-wide K chunks staged in shared memory.
constexpr int kFoldK = 32;
template <typename T>
constexpr size_t fold_smem() {
  return sizeof(T) * 2 * (size_t)NB * (kFoldK + 1);
}
template <typename T>
static __global__ void __launch_bounds__(256) fold_kernel(const T* __restrict__ S, int ld, const T* __restrict__ Linv,
                                                          int ntiles, T* __restrict__ Mf, T* __restrict__ Pb,
                                                          const int* __restrict__ active) {
  extern __shared__ __align__(16) unsigned char fsm[];
  T* As = reinterpret_cast<T*>(fsm);  // NB x (kFoldK + 1): A(i, m)
  T* Bs = As + NB * (kFoldK + 1);     // kFoldK x ... stored as NB x (kFoldK + 1): B(m, j) at j (kFoldK + 1) + m
  if (active && !*active) return;
  const int nf = ntiles - 1;
  const bool fwd = (int)blockIdx.x < nf;
  const int I = fwd ? (int)blockIdx.x + 1 : (int)blockIdx.x - nf;
  // A(i, m) = a0[i * ai + m * am], B(m, j) = b0[m * bm + j * bj]
  const T* Li = Linv + (size_t)I * NB * NB;
  const T* a0;
  const T* b0;
  size_t ai, am, bm, bj;
  if (fwd) {  // inv(L_II) x L_I,I-1
    a0 = Li;
    ai = NB;
    am = 1;
    b0 = S + (size_t)I * NB * ld + (size_t)(I - 1) * NB;
    bm = (size_t)ld;
    bj = 1;
  } else {  // inv(L_II)' x L_I+1,I'
    a0 = Li;
    ai = 1;
    am = NB;
    b0 = S + (size_t)(I + 1) * NB * ld + (size_t)I * NB;
    bm = 1;
    bj = (size_t)ld;
  }
  T* out = (fwd ? Mf : Pb) + (size_t)I * NB * NB;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  T acc[8][8];
#pragma unroll
  for (int u = 0; u < 8; u++)
#pragma unroll
    for (int v = 0; v < 8; v++) acc[u][v] = (T)0;
  for (int k0 = 0; k0 < NB; k0 += kFoldK) {
    for (int e = tid; e < NB * kFoldK; e += 256) {
      const int r = e / kFoldK, m = e - (e / kFoldK) * kFoldK;
      As[r * (kFoldK + 1) + m] = a0[(size_t)r * ai + (size_t)(k0 + m) * am];
      Bs[r * (kFoldK + 1) + m] = b0[(size_t)(k0 + m) * bm + (size_t)r * bj];
    }
    __syncthreads();
#pragma unroll 4
    for (int m = 0; m < kFoldK; m++) {
      T a[8], b[8];
#pragma unroll
      for (int u = 0; u < 8; u++) a[u] = As[(ty + 16 * u) * (kFoldK + 1) + m];
#pragma unroll
      for (int v = 0; v < 8; v++) b[v] = Bs[(tx + 16 * v) * (kFoldK + 1) + m];
#pragma unroll
      for (int u = 0; u < 8; u++)
#pragma unroll
        for (int v = 0; v < 8; v++) acc[u][v] += a[u] * b[v];
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 8; u++)
#pragma unroll
    for (int v = 0; v < 8; v++) out[(size_t)(ty + 16 * u) * NB + tx + 16 * v] = acc[u][v];
}

// Forward: y = L^-1 b.  512 threads; warp w owns rows 8 w .. 8 w + 7 of the
// CTA's tile, lane l columns 4 l .. 4 l + 3.
template <typename T>
static __global__ void __launch_bounds__(SV) trsv_fwd_fold_kernel(const T* __restrict__ L, int ld, int ntiles,
                                                                  const T* __restrict__ Linv,
                                                                  const T* __restrict__ Mf,
                                                                  const double* __restrict__ b, double* y,
                                                                  int* __restrict__ ticket, int* __restrict__ status,
                                                                  long long limit, const int* __restrict__ env,
                                                                  const int* __restrict__ active) {
  extern __shared__ float4 sLi4[];
  T* sLi = reinterpret_cast<T*>(sLi4);  // inv(L_II), NB x NB
  __shared__ double acc[NB];
  __shared__ int I_s;
  if (active && !*active) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) I_s = atomicAdd(ticket, 1);
  __syncthreads();
  const int I = I_s;
  {
    const float4* src = reinterpret_cast<const float4*>(Linv + (size_t)I * NB * NB);
    for (int i = tid; i < (int)(NB * NB * sizeof(T) / 16); i += SV) sLi4[i] = src[i];
  }
  const int J0 = env ? env[I] : 0;
  const bool fold = I - 1 >= J0;
  double part[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  bool ok = true;
  const T* Lrow = L + (size_t)(I * NB + warp * 8) * ld + 4 * lane;
  for (int J = J0; J < I - 1; J++) {
    double lv[8][4];  // the L tile does not depend on y_J: load it before waiting
#pragma unroll
    for (int rr = 0; rr < 8; rr++) load4(Lrow + (size_t)rr * ld + (size_t)J * NB, lv[rr]);
    double yv[4];
    const bool got = wait_values4(y + (size_t)J * NB + 4 * lane, yv, limit);
    if (!__all_sync(0xffffffffu, got)) {
      ok = false;
      break;
    }
#pragma unroll
    for (int rr = 0; rr < 8; rr++)
      part[rr] += lv[rr][0] * yv[0] + lv[rr][1] * yv[1] + lv[rr][2] * yv[2] + lv[rr][3] * yv[3];
  }
  // the folded tile M_I (this thread's 8 rows x 4 columns): its loads overlap
  // the reductions below and the wait for y_{I-1}
  double mv[8][4];
  if (fold) {
    const T* Mr = Mf + (size_t)I * NB * NB + (size_t)(warp * 8) * NB + 4 * lane;
#pragma unroll
    for (int rr = 0; rr < 8; rr++) load4(Mr + (size_t)rr * NB, mv[rr]);
  }
#pragma unroll
  for (int rr = 0; rr < 8; rr++) {
    const double s = warp_sum(part[rr]);
    if (lane == 0) acc[warp * 8 + rr] = b[(size_t)I * NB + warp * 8 + rr] - s;
  }
  __syncthreads();
  // c_I = inv(L_II) acc, every lane holding all 8 of its warp's rows
  const T* Li = sLi + (size_t)(warp * 8) * NB + 4 * lane;
  const double av[4] = {acc[4 * lane], acc[4 * lane + 1], acc[4 * lane + 2], acc[4 * lane + 3]};
  double c[8];
#pragma unroll
  for (int rr = 0; rr < 8; rr++) {
    double lv[4];
    load4(Li + (size_t)rr * NB, lv);
    c[rr] = warp_all_sum_d(lv[0] * av[0] + lv[1] * av[1] + lv[2] * av[2] + lv[3] * av[3]);
  }
  if (fold && ok) {
    double yv[4];
    ok = __all_sync(0xffffffffu, wait_values4(y + (size_t)(I - 1) * NB + 4 * lane, yv, limit));
#pragma unroll
    for (int rr = 0; rr < 8; rr++)
      c[rr] -= warp_all_sum_d(mv[rr][0] * yv[0] + mv[rr][1] * yv[1] + mv[rr][2] * yv[2] + mv[rr][3] * yv[3]);
  }
  if (__all_sync(0xffffffffu, ok)) {
#pragma unroll
    for (int rr = 0; rr < 8; rr++)
      if (lane == rr) st_relaxed_f64(y + (size_t)I * NB + warp * 8 + rr, c[rr]);
  } else if (lane == 0) {
    atomicOr(status, ST_SPIN_TIMEOUT);
  }
}

// Backward: x = L'^-1 y.  Warp w owns output columns 8 w .. 8 w + 7 of the
// folded step and rows 8 w .. of the L tiles of the sum; lane l columns / rows
// 4 l .. 4 l + 3.
template <typename T>
static __global__ void __launch_bounds__(SV) trsv_bwd_fold_kernel(const T* __restrict__ L, int ld, int ntiles,
                                                                  const T* __restrict__ Linv,
                                                                  const T* __restrict__ Pb,
                                                                  const double* __restrict__ yv_in, double* x,
                                                                  int* __restrict__ ticket, int* __restrict__ status,
                                                                  long long limit, const int* __restrict__ env,
                                                                  const int* __restrict__ active) {
  extern __shared__ float4 sLi4[];
  T* sLiT = reinterpret_cast<T*>(sLi4);  // inv(L_II) transposed: sLiT[c][r] = Linv[r][c]
  __shared__ double red[SV / 32][NB];
  __shared__ double acc[NB];
  __shared__ int I_s;
  if (active && !*active) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) I_s = ntiles - 1 - atomicAdd(ticket, 1);
  __syncthreads();
  const int I = I_s;
  {
    const T* src = Linv + (size_t)I * NB * NB;
    for (int i = tid; i < NB * NB; i += SV) {
      const int r = i / NB, cc = i - (i / NB) * NB;
      sLiT[cc * NB + r] = src[i];
    }
  }
  const int Jlast = env ? env[ntiles + I] : ntiles - 1;
  const bool fold = Jlast >= I + 1;
  double part[4] = {0, 0, 0, 0};
  bool ok = true;
  for (int J = Jlast; J > I + 1; J--) {
    const T* Lb = L + (size_t)(J * NB + warp * 8) * ld + (size_t)I * NB + 4 * lane;
    double lv[8][4];  // loaded before waiting for x_J
#pragma unroll
    for (int rr = 0; rr < 8; rr++) load4(Lb + (size_t)rr * ld, lv[rr]);
    // x_J rows 8 w .. 8 w + 7: lanes 0..1 poll four each, then broadcast
    double xq[4] = {0, 0, 0, 0};
    bool got = true;
    if (lane < 2) got = wait_values4(x + (size_t)J * NB + warp * 8 + 4 * lane, xq, limit);
    if (!__all_sync(0xffffffffu, got)) {
      ok = false;
      break;
    }
#pragma unroll
    for (int rr = 0; rr < 8; rr++) {
      const double xr = __shfl_sync(0xffffffffu, xq[rr & 3], rr >> 2);
      part[0] += lv[rr][0] * xr;
      part[1] += lv[rr][1] * xr;
      part[2] += lv[rr][2] * xr;
      part[3] += lv[rr][3] * xr;
    }
  }
  // the folded tile P_I: loads overlap the reductions and the wait for x_{I+1}
  double pv[8][4];
  if (fold) {
    const T* Pr = Pb + (size_t)I * NB * NB + (size_t)(warp * 8) * NB + 4 * lane;
#pragma unroll
    for (int rr = 0; rr < 8; rr++) load4(Pr + (size_t)rr * NB, pv[rr]);
  }
#pragma unroll
  for (int q = 0; q < 4; q++) red[warp][4 * lane + q] = part[q];
  __syncthreads();
  if (tid < NB) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < SV / 32; w++) s += red[w][tid];
    acc[tid] = yv_in[(size_t)I * NB + tid] - s;
  }
  __syncthreads();
  // d_I = inv(L_II)' acc: output c = 8 w + rr, lanes over rows r = 4 l ..
  const double av[4] = {acc[4 * lane], acc[4 * lane + 1], acc[4 * lane + 2], acc[4 * lane + 3]};
  double dv[8];
#pragma unroll
  for (int rr = 0; rr < 8; rr++) {
    double lt[4];
    load4(sLiT + (size_t)(warp * 8 + rr) * NB + 4 * lane, lt);
    dv[rr] = warp_all_sum_d(lt[0] * av[0] + lt[1] * av[1] + lt[2] * av[2] + lt[3] * av[3]);
  }
  if (fold && ok) {
    double xv[4];
    ok = __all_sync(0xffffffffu, wait_values4(x + (size_t)(I + 1) * NB + 4 * lane, xv, limit));
#pragma unroll
    for (int rr = 0; rr < 8; rr++)
      dv[rr] -= warp_all_sum_d(pv[rr][0] * xv[0] + pv[rr][1] * xv[1] + pv[rr][2] * xv[2] + pv[rr][3] * xv[3]);
  }
  if (__all_sync(0xffffffffu, ok)) {
#pragma unroll
    for (int rr = 0; rr < 8; rr++)
      if (lane == rr) st_relaxed_f64(x + (size_t)I * NB + warp * 8 + rr, dv[rr]);
  } else if (lane == 0) {
    atomicOr(status, ST_SPIN_TIMEOUT);
  }
}

}  // namespace nl
