// cholesky.cuh -- blocked right-looking Cholesky of the reduced camera system.
//
// Replaces the dense LDLT factorisation + solve of SolverCholeskySchur
// (SolverCholeskyEigenDense::factorize/solve, nelson/SolverCholeskyDense.hpp:15-24,
// used at nelson/SolverCholeskySchur.hpp:136-140).  S is stored dense,
// row-major, lower triangle, n padded to a multiple of NB = 128 (identity on
// the padding).  Per 128-wide panel k:
//   potrf_diag_kernel  FP64 factor of the diagonal tile and its inverse (one CTA)
//   trsm_kernel        L_ik = A_ik L_kk^-T as a product with the inverse
//   syrk update        A_ij -= L_ik L_jk' on the trailing lower triangle
//                      (tensor-core kernel in tc_syrk.cu for the mixed path,
//                      cuBLAS DSYRK for the FP64 comparison path)
// Solves use the tile inverses: trsv_fwd/bwd_kernel with a ticketed
// look-back between CTAs of one launch, each wait bounded.
#pragma once

#include "nl_common.cuh"

namespace nl {

constexpr int NB = 128;
constexpr long long kSpinLimit = 1LL << 24;  // bounded waits (~1 s worst case)

// ---------------------------------------------------------------------------
// One CTA: factor the NB x NB diagonal tile of panel k in FP64 shared memory
// (32-wide sub-panels: warp-register factor of the 32x32 diagonal,
// substitution for the rows below, rank-32 update), write L_kk back to S and
// inv(L_kk) (FP64, full NB x NB with zeros above the diagonal) to Linv.
template <typename T>
static __global__ void __launch_bounds__(256) potrf_diag_kernel(T* __restrict__ S, int ld, int k,
                                                          double* __restrict__ Linv, int* __restrict__ status,
                                                          const int* __restrict__ active) {
  extern __shared__ double sA[];  // NB x (NB + 1)
  constexpr int LDS = NB + 1;
  if (active && !*active) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t base = (size_t)k * NB * ld + (size_t)k * NB;
  for (int i = tid; i < NB * NB; i += 256) {
    const int r = i / NB, c = i - r * NB;
    sA[r * LDS + c] = c <= r ? (double)S[base + (size_t)r * ld + c] : 0.0;
  }
  __syncthreads();
  __shared__ int bad;
  if (tid == 0) bad = 0;
  __syncthreads();
  for (int s = 0; s < NB / 32; s++) {
    const int c0 = 32 * s;
    if (warp == 0) {
      double a[32];
#pragma unroll
      for (int j = 0; j < 32; j++) a[j] = (j <= lane) ? sA[(c0 + lane) * LDS + c0 + j] : 0.0;
      bool fail = false;
#pragma unroll
      for (int j = 0; j < 32; j++) {
        const double piv = __shfl_sync(0xffffffffu, a[j], j);
        fail |= !(piv > 0.0) || !isfinite(piv);
        const double dj = sqrt(fmax(piv, 1e-300));
        const double inv = 1.0 / dj;
        if (lane == j) a[j] = dj;
        else if (lane > j) a[j] *= inv;
#pragma unroll
        for (int l = j + 1; l < 32; l++) {
          const double llj = __shfl_sync(0xffffffffu, a[j], l);
          if (lane >= l) a[l] -= a[j] * llj;
        }
      }
#pragma unroll
      for (int j = 0; j < 32; j++)
        if (j <= lane) sA[(c0 + lane) * LDS + c0 + j] = a[j];
      if (fail && lane == 0) bad = 1;
    }
    __syncthreads();
    // rows below: X = A * L_ss^-T by substitution (one row per thread)
    for (int r = c0 + 32 + tid; r < NB; r += 256) {
      double x[32];
#pragma unroll
      for (int j = 0; j < 32; j++) x[j] = sA[r * LDS + c0 + j];
#pragma unroll
      for (int j = 0; j < 32; j++) {
        double v = x[j];
#pragma unroll
        for (int l = 0; l < j; l++) v -= x[l] * sA[(c0 + j) * LDS + c0 + l];
        x[j] = v / sA[(c0 + j) * LDS + c0 + j];
      }
#pragma unroll
      for (int j = 0; j < 32; j++) sA[r * LDS + c0 + j] = x[j];
    }
    __syncthreads();
    // trailing update inside the tile: rows/cols [c0 + 32, NB), lower
    const int m = NB - c0 - 32;
    const int cnt = m * (m + 1) / 2;
    for (int idx = tid; idx < cnt; idx += 256) {
      int r = (int)((sqrt(8.0 * idx + 1.0) - 1.0) * 0.5);
      while ((r + 1) * (r + 2) / 2 <= idx) r++;
      while (r * (r + 1) / 2 > idx) r--;
      const int c = idx - r * (r + 1) / 2;
      const int R = c0 + 32 + r, Cc = c0 + 32 + c;
      double v = sA[R * LDS + Cc];
#pragma unroll 8
      for (int l = 0; l < 32; l++) v -= sA[R * LDS + c0 + l] * sA[Cc * LDS + c0 + l];
      sA[R * LDS + Cc] = v;
    }
    __syncthreads();
  }
  if (tid == 0 && bad) atomicOr(status, ST_CHOL_FAIL);
  // write L back
  for (int i = tid; i < NB * NB; i += 256) {
    const int r = i / NB, c = i - r * NB;
    if (c <= r) S[base + (size_t)r * ld + c] = (T)sA[r * LDS + c];
  }
  // inverse, column c by thread c: L x = e_c; x kept in the (unused) upper
  // triangle of sA, row c: sA[c][i] = Linv[i][c] for i > c.
  __syncthreads();
  double* out = Linv + (size_t)k * NB * NB;
  if (tid < NB) {
    const int c = tid;
    const double dc = 1.0 / sA[c * LDS + c];
    for (int i = c + 1; i < NB; i++) {
      double v = sA[i * LDS + c] * dc;
      for (int l = c + 1; l < i; l++) v += sA[i * LDS + l] * sA[c * LDS + l];
      sA[c * LDS + i] = -v / sA[i * LDS + i];
    }
    // column c of Linv
    for (int i = 0; i < NB; i++) {
      double v = 0.0;
      if (i == c) v = dc;
      else if (i > c) v = sA[c * LDS + i];
      out[(size_t)i * NB + c] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// L_ik = A_ik inv(L_kk)' for 32-row slabs below the diagonal tile.
// Thread j computes column j of the slab: X[r][j] = sum_{l<=j} A[r][l] Linv[j][l].
template <typename T>
static __global__ void __launch_bounds__(NB) trsm_kernel(T* __restrict__ S, int ld, int k, int nrows_below,
                                                  const double* __restrict__ Linv, const int* __restrict__ active) {
  extern __shared__ unsigned char smraw[];
  T* sL = reinterpret_cast<T*>(smraw);  // NB x (NB + 1), Linv in T
  T* sX = sL + NB * (NB + 1);            // 32 x NB rows of A
  if (active && !*active) return;
  const int tid = threadIdx.x;
  const int r0 = (k + 1) * NB + blockIdx.x * 32;
  const int nr = min(32, (k + 1) * NB + nrows_below - r0);
  if (nr <= 0) return;
  const double* Li = Linv + (size_t)k * NB * NB;
  for (int i = tid; i < NB * NB; i += NB) {
    const int r = i / NB, c = i - r * NB;
    sL[r * (NB + 1) + c] = (T)Li[i];
  }
  for (int i = tid; i < 32 * NB; i += NB) {
    const int r = i / NB, c = i - r * NB;
    sX[i] = r < nr ? S[(size_t)(r0 + r) * ld + (size_t)k * NB + c] : (T)0;
  }
  __syncthreads();
  const int j = tid;
  T acc[32];
#pragma unroll
  for (int r = 0; r < 32; r++) acc[r] = (T)0;
  for (int l = 0; l <= j; l++) {
    const T lj = sL[j * (NB + 1) + l];
#pragma unroll
    for (int r = 0; r < 32; r++) acc[r] += sX[r * NB + l] * lj;
  }
  __syncthreads();
  for (int r = 0; r < nr; r++) S[(size_t)(r0 + r) * ld + (size_t)k * NB + j] = acc[r];
}

// ---------------------------------------------------------------------------
// CUDA-core trailing update (FP32 or FP64), one CTA per 128 x 128 lower tile:
// C_IJ -= X_I X_J' with X = columns [k NB, (k+1) NB).  Used as the portable
// reference of the tensor-core kernel and for small problems.
template <typename T>
static __global__ void __launch_bounds__(256) syrk_cc_kernel(T* __restrict__ S, int ld, int k, int t0, int nt,
                                                      const int* __restrict__ active) {
  constexpr int KC = 16;
  __shared__ T As[KC][NB + 4];
  __shared__ T Bs[KC][NB + 4];
  if (active && !*active) return;
  const int q = blockIdx.x;
  int I = (int)((sqrt(8.0 * q + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= q) I++;
  while (I * (I + 1) / 2 > q) I--;
  const int J = q - I * (I + 1) / 2;
  const int rA = (t0 + I) * NB, rB = (t0 + J) * NB, kc = k * NB;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = (T)0;
  for (int kk = 0; kk < NB; kk += KC) {
    for (int i = threadIdx.x; i < NB * KC; i += 256) {
      const int r = i / KC, c = i - r * KC;
      As[c][r] = S[(size_t)(rA + r) * ld + kc + kk + c];
      Bs[c][r] = S[(size_t)(rB + r) * ld + kc + kk + c];
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < KC; c++) {
      T a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = As[c][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 8; j++) b[j] = Bs[c][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int r = ty + 16 * i;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = tx + 16 * j;
      if (I != J || c <= r) S[(size_t)(rA + r) * ld + rB + c] -= acc[i][j];
    }
  }
}

// ---------------------------------------------------------------------------
// Triangular solves with the tile inverses.  CTAs take tickets in tile order
// (forward) or reverse order (backward); a CTA only waits on tiles whose
// owners took earlier tickets, so every wait ends; each wait is also bounded.
static __device__ inline bool wait_flag(const int* flag, int epoch, int* status) {
  long long it = 0;
  while (*(volatile const int*)flag != epoch) {
    if (++it > kSpinLimit) {
      atomicOr(status, ST_SPIN_TIMEOUT);
      return false;
    }
    __nanosleep(32);
  }
  __threadfence();
  return true;
}

template <typename T>
static __global__ void __launch_bounds__(256) trsv_fwd_kernel(const T* __restrict__ L, int ld, int ntiles,
                                                       const double* __restrict__ Linv, const double* __restrict__ b,
                                                       double* __restrict__ y, int* __restrict__ ticket,
                                                       int* __restrict__ flags, int epoch, int* __restrict__ status,
                                                       const int* __restrict__ active) {
  __shared__ double acc[NB];
  __shared__ double yj[NB];
  __shared__ int I_s, ok_s;
  if (active && !*active) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) I_s = atomicAdd(ticket, 1);
  __syncthreads();
  const int I = I_s;
  if (tid < NB) acc[tid] = b[(size_t)I * NB + tid];
  __syncthreads();
  for (int J = 0; J < I; J++) {
    if (tid == 0) ok_s = wait_flag(flags + J, epoch, status) ? 1 : 0;
    __syncthreads();
    if (!ok_s) return;
    if (tid < NB) yj[tid] = ((volatile double*)y)[(size_t)J * NB + tid];
    __syncthreads();
    // rows r = warp*16 .. +15: acc[r] -= L[I*NB + r][J*NB ...] . yj
    for (int rr = 0; rr < 16; rr++) {
      const int r = warp * 16 + rr;
      const T* row = L + (size_t)(I * NB + r) * ld + (size_t)J * NB;
      double s = 0.0;
#pragma unroll
      for (int c = lane; c < NB; c += 32) s += (double)row[c] * yj[c];
      s = warp_sum(s);
      if (lane == 0) acc[r] -= s;
    }
    __syncthreads();
  }
  // y_I = Linv_I acc
  const double* Li = Linv + (size_t)I * NB * NB;
  for (int rr = 0; rr < 16; rr++) {
    const int r = warp * 16 + rr;
    double s = 0.0;
#pragma unroll
    for (int c = lane; c < NB; c += 32) s += Li[(size_t)r * NB + c] * acc[c];
    s = warp_sum(s);
    if (lane == 0) y[(size_t)I * NB + r] = s;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) atomicExch(flags + I, epoch);
}

template <typename T>
static __global__ void __launch_bounds__(256) trsv_bwd_kernel(const T* __restrict__ L, int ld, int ntiles,
                                                       const double* __restrict__ Linv, const double* __restrict__ yv,
                                                       double* __restrict__ x, int* __restrict__ ticket,
                                                       int* __restrict__ flags, int epoch, int* __restrict__ status,
                                                       const int* __restrict__ active) {
  __shared__ double acc[2][NB];
  __shared__ double xj[NB];
  __shared__ int I_s, ok_s;
  if (active && !*active) return;
  const int tid = threadIdx.x;
  if (tid == 0) I_s = ntiles - 1 - atomicAdd(ticket, 1);
  __syncthreads();
  const int I = I_s;
  const int c = tid & (NB - 1), half = tid >> 7;  // 2 threads per column
  acc[half][c] = half == 0 ? yv[(size_t)I * NB + c] : 0.0;
  for (int J = ntiles - 1; J > I; J--) {
    if (tid == 0) ok_s = wait_flag(flags + J, epoch, status) ? 1 : 0;
    __syncthreads();
    if (!ok_s) return;
    if (tid < NB) xj[tid] = ((volatile double*)x)[(size_t)J * NB + tid];
    __syncthreads();
    // acc[c] -= sum_r L[J*NB + r][I*NB + c] xj[r]
    double s = 0.0;
    for (int r = half * 64; r < half * 64 + 64; r++) s += (double)L[(size_t)(J * NB + r) * ld + (size_t)I * NB + c] * xj[r];
    acc[half][c] -= s;
    __syncthreads();
  }
  __syncthreads();
  if (tid < NB) acc[0][tid] += acc[1][tid];
  __syncthreads();
  // x_I = Linv_I' acc : x[c] = sum_r Linv[r][c] acc[r]
  const double* Li = Linv + (size_t)I * NB * NB;
  if (tid < NB) {
    double s = 0.0;
    for (int r = 0; r < NB; r++) s += Li[(size_t)r * NB + tid] * acc[0][r];
    x[(size_t)I * NB + tid] = s;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) atomicExch(flags + I, epoch);
}

// ---------------------------------------------------------------------------
// Refinement residual r = b - S0 x from the lower storage of S0, in two
// passes: partial products per (row tile, chunk), then a fixed-order sum.
// Row r of S0 is (lower row r) + (column r below the diagonal).
template <typename T, int NCH>
static __global__ void __launch_bounds__(NB) symv_partial_kernel(const T* __restrict__ S0, int ld, int n_pad,
                                                          const double* __restrict__ x, double* __restrict__ part,
                                                          const int* __restrict__ active) {
  if (active && !*active) return;
  const int I = blockIdx.x, ch = blockIdx.y;
  const int r = threadIdx.x;
  const int R = I * NB + r;
  // this chunk's slice of columns [c0, c1)
  const int per = (n_pad + NCH - 1) / NCH;
  const int c0 = ch * per, c1 = min(n_pad, c0 + per);
  double s = 0.0;
  // lower part of row R: columns c <= R -> S0[R][c]; upper part c > R -> S0[c][R]
  // lower: thread r walks its own row (uncoalesced across threads, but rows are
  // read once); upper: coalesced over r.
  const int lo_end = min(c1, R + 1);
  for (int c = c0; c < lo_end; c++) s += (double)S0[(size_t)R * ld + c] * x[c];
  for (int c = max(c0, R + 1); c < c1; c++) s += (double)S0[(size_t)c * ld + R] * x[c];
  part[(size_t)ch * n_pad + R] = s;
}

template <int NCH>
static __global__ void resid_finalize_kernel(const double* __restrict__ part, const double* __restrict__ b, int n_pad,
                                      double* __restrict__ r, const int* __restrict__ active) {
  if (active && !*active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pad) return;
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < NCH; c++) s += part[(size_t)c * n_pad + i];
  r[i] = b[i] - s;
}

static __global__ void axpy_kernel(double* __restrict__ x, const double* __restrict__ d, int n,
                            const int* __restrict__ active) {
  if (active && !*active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += d[i];
}

}  // namespace nl
