// potrf_blocked.cuh -- FP32 factor and inverse of one 128 x 128 diagonal tile
// as a 4 x 4 block recursion over 32 x 32 blocks (the mixed path's critical
// chain: every panel of the reduced-camera-system Cholesky waits for it).
//
// For block column kb = 0 .. 3 (K0 = 32 kb):
//   warp 0   factors the 32 x 32 diagonal block in registers (lane i holds row
//            i; column j's pivot and entries are exchanged by warp shuffles)
//            and inverts its factor the same way (lane i builds row i of
//            X = inv(L) by forward substitution, rows finalised in order);
//   TRSM     L_ik = A_ik X_kk' for the blocks below, two warps per block;
//   update   A_ij -= L_ik L_jk' for kb < j <= i, two warps per block, reading
//            the new panel from a transposed copy so a warp's lanes read
//            consecutive words.
// Then the off-diagonal blocks of inv(L), by distance d = i - j from the
// diagonal: T = sum_{m=j}^{i-1} L_im X_mj, X_ij = -X_ii T.
// Every product is a 4 x 4 register tile per lane (a warp covers 16 rows x 32
// columns of a block), operands in shared memory read as 16-byte vectors:
// rows of the left operand are the same for eight lanes (broadcast), the right
// operand's columns run across the lanes.  The work on the critical path is 4
// sequential 32-wide block steps instead of 32 sequential rank-4 steps.
// L goes to S (zeros above its diagonal) and the blocks of inv(L) on and below
// the diagonal to Linv (its strictly upper blocks are never written: the
// caller keeps them zero).  A non-positive pivot sets ST_CHOL_FAIL.
#pragma once

#include "cholesky.cuh"

namespace nl {

constexpr int kPB = 32;                     // block width
constexpr int kPLD = NB + 4;                // row stride of the 128-wide buffers (floats)
constexpr int kTLD = kPB + 4;               // row stride of the 32-wide buffers
constexpr int kPotrf32Threads = 512;
constexpr size_t kPotrf32Smem =
    sizeof(float) * ((size_t)2 * NB * kPLD + (size_t)kPB * kPLD + (size_t)kPB * kTLD + (size_t)3 * kPB * kTLD);

// acc[u][v] += sum_{m < K} A[(r0 + u) lda + m] B[m ldb + c0 + v]   (K % 4 == 0)
__device__ __forceinline__ void tile4x4(const float* __restrict__ A, int lda, const float* __restrict__ B, int ldb,
                                        int K, int r0, int c0, float acc[4][4]) {
#pragma unroll 2
  for (int m = 0; m < K; m += 4) {
    float4 a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; u++) a[u] = *reinterpret_cast<const float4*>(A + (size_t)(r0 + u) * lda + m);
#pragma unroll
    for (int q = 0; q < 4; q++) b[q] = *reinterpret_cast<const float4*>(B + (size_t)(m + q) * ldb + c0);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const float av[4] = {a[u].x, a[u].y, a[u].z, a[u].w};
#pragma unroll
      for (int q = 0; q < 4; q++) {
        acc[u][0] += av[q] * b[q].x;
        acc[u][1] += av[q] * b[q].y;
        acc[u][2] += av[q] * b[q].z;
        acc[u][3] += av[q] * b[q].w;
      }
    }
  }
}

static __global__ void __launch_bounds__(kPotrf32Threads) potrf32_kernel(float* __restrict__ S, int ld, int k,
                                                                         float* __restrict__ Linv,
                                                                         int* __restrict__ status,
                                                                         const int* __restrict__ active) {
  extern __shared__ __align__(16) float sm[];
  float* As = sm;                    // NB x kPLD: the tile, A -> L in place (lower part)
  float* Xs = As + NB * kPLD;        // NB x kPLD: inv(L) (lower blocks)
  float* PT = Xs + NB * kPLD;        // kPB x kPLD: the new panel transposed, PT[m][row] = L[row][K0 + m]
  float* XkT = PT + kPB * kPLD;      // kPB x kTLD: X_kk transposed
  float* Tb = XkT + kPB * kTLD;      // 3 x kPB x kTLD: products of the inverse assembly
  chain_release();
  chain_wait();
  if (active && !*active) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned FULL = 0xffffffffu;
  const size_t base = (size_t)k * NB * ld + (size_t)k * NB;
  // load the tile (16-byte vectors; entries above the diagonal are never used)
  for (int i = tid; i < NB * NB / 4; i += kPotrf32Threads) {
    const int r = i >> 5, c = (i & 31) * 4;
    *reinterpret_cast<float4*>(As + r * kPLD + c) = *reinterpret_cast<const float4*>(S + base + (size_t)r * ld + c);
  }
  __syncthreads();
  // lane tile of a 32 x 32 block within a warp pair: rows 16 sub + 4 (lane >> 3), columns 4 (lane & 7)
  const int rq = 4 * (lane >> 3), c0 = 4 * (lane & 7);
  for (int kb = 0; kb < 4; kb++) {
    const int K0 = kPB * kb;
    if (warp == 0) {
      float a[kPB];
      const float* rowp = As + (K0 + lane) * kPLD + K0;
#pragma unroll
      for (int c = 0; c < kPB; c += 4) {
        const float4 v = *reinterpret_cast<const float4*>(rowp + c);
        a[c] = v.x;
        a[c + 1] = v.y;
        a[c + 2] = v.z;
        a[c + 3] = v.w;
      }
      bool bad = false;
      float myrs = 0.f;  // 1 / L_ii of this lane's row
#pragma unroll
      for (int j = 0; j < kPB; j++) {
        const float d = __shfl_sync(FULL, a[j], j);
        bad |= !(d > 0.f) || !isfinite(d);
        const float rs = pivot_rsqrt(d);
        if (lane == j) {
          a[j] = d * rs;
          myrs = rs;
        } else if (lane > j) {
          a[j] *= rs;
        }
#pragma unroll
        for (int c = j + 1; c < kPB; c++) {
          const float lcj = __shfl_sync(FULL, a[j], c);
          if (lane >= c) a[c] -= a[j] * lcj;
        }
      }
      // X = inv(L_kk), row `lane`: rows finalised in order, multiplications only
      float x[kPB];
#pragma unroll
      for (int c = 0; c < kPB; c++) x[c] = 0.f;
#pragma unroll
      for (int kk = 0; kk < kPB; kk++) {
        const float rk = __shfl_sync(FULL, myrs, kk);
        if (lane == kk) {
#pragma unroll
          for (int c = 0; c <= kk; c++) x[c] = ((c == kk ? 1.f : 0.f) - x[c]) * rk;
        }
#pragma unroll
        for (int c = 0; c <= kk; c++) {
          const float xkc = __shfl_sync(FULL, x[c], kk);
          if (lane > kk) x[c] += a[kk] * xkc;
        }
      }
      float* lrow = As + (K0 + lane) * kPLD + K0;
      float* xrow = Xs + (K0 + lane) * kPLD + K0;
#pragma unroll
      for (int c = 0; c < kPB; c += 4) {
        *reinterpret_cast<float4*>(lrow + c) =
            make_float4(c <= lane ? a[c] : 0.f, c + 1 <= lane ? a[c + 1] : 0.f, c + 2 <= lane ? a[c + 2] : 0.f,
                        c + 3 <= lane ? a[c + 3] : 0.f);
        *reinterpret_cast<float4*>(xrow + c) = make_float4(x[c], x[c + 1], x[c + 2], x[c + 3]);
      }
#pragma unroll
      for (int c = 0; c < kPB; c++) XkT[c * kTLD + lane] = x[c];
      if (__any_sync(FULL, bad) && lane == 0) atomicOr(status, ST_CHOL_FAIL);
    }
    __syncthreads();
    // TRSM: L_ik = A_ik X_kk' for the blocks below (two warps per block)
    const int nblk = 3 - kb;
    if (warp < 2 * nblk) {
      const int bi = kb + 1 + (warp >> 1), r0 = 16 * (warp & 1) + rq;
      float acc[4][4] = {};
      tile4x4(As + (size_t)(kPB * bi) * kPLD + K0, kPLD, XkT, kTLD, kPB, r0, c0, acc);
      __syncwarp();  // the lanes sharing these rows have read them
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int row = kPB * bi + r0 + u;
        *reinterpret_cast<float4*>(As + (size_t)row * kPLD + K0 + c0) =
            make_float4(acc[u][0], acc[u][1], acc[u][2], acc[u][3]);
#pragma unroll
        for (int v = 0; v < 4; v++) PT[(c0 + v) * kPLD + row] = acc[u][v];
      }
    }
    __syncthreads();
    // trailing update A_ij -= L_ik L_jk', kb < j <= i (two warps per block)
    const int npair = nblk * (nblk + 1) / 2;
    if (warp < 2 * npair) {
      int pi = warp >> 1, bi = kb + 1, bj = kb + 1;
      while (pi > bi - (kb + 1)) {
        pi -= bi - kb;
        bi++;
      }
      bj = kb + 1 + pi;
      const int r0 = 16 * (warp & 1) + rq;
      float acc[4][4] = {};
      tile4x4(As + (size_t)(kPB * bi) * kPLD + K0, kPLD, PT + kPB * bj, kPLD, kPB, r0, c0, acc);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        float* p = As + (size_t)(kPB * bi + r0 + u) * kPLD + kPB * bj + c0;
        float4 v = *reinterpret_cast<float4*>(p);
        v.x -= acc[u][0];
        v.y -= acc[u][1];
        v.z -= acc[u][2];
        v.w -= acc[u][3];
        *reinterpret_cast<float4*>(p) = v;
      }
    }
    __syncthreads();
  }
  // off-diagonal blocks of inv(L) by distance d from the diagonal
  for (int d = 1; d < 4; d++) {
    const int nb = 4 - d;
    if (warp < 2 * nb) {
      const int j = warp >> 1, i = j + d, r0 = 16 * (warp & 1) + rq;
      float acc[4][4] = {};
      // T = sum_{m=j}^{i-1} L_im X_mj
      tile4x4(As + (size_t)(kPB * i) * kPLD + kPB * j, kPLD, Xs + (size_t)(kPB * j) * kPLD + kPB * j, kPLD, kPB * d,
              r0, c0, acc);
      float* T = Tb + (size_t)j * kPB * kTLD;
#pragma unroll
      for (int u = 0; u < 4; u++)
        *reinterpret_cast<float4*>(T + (r0 + u) * kTLD + c0) = make_float4(acc[u][0], acc[u][1], acc[u][2], acc[u][3]);
    }
    __syncthreads();
    if (warp < 2 * nb) {
      const int j = warp >> 1, i = j + d, r0 = 16 * (warp & 1) + rq;
      float acc[4][4] = {};
      tile4x4(Xs + (size_t)(kPB * i) * kPLD + kPB * i, kPLD, Tb + (size_t)j * kPB * kTLD, kTLD, kPB, r0, c0, acc);
#pragma unroll
      for (int u = 0; u < 4; u++)
        *reinterpret_cast<float4*>(Xs + (size_t)(kPB * i + r0 + u) * kPLD + kPB * j + c0) =
            make_float4(-acc[u][0], -acc[u][1], -acc[u][2], -acc[u][3]);
    }
    __syncthreads();
  }
  // write L (zeros above its diagonal) and the lower blocks of inv(L)
  float* Lout = Linv + (size_t)k * NB * NB;
  for (int i = tid; i < NB * NB / 4; i += kPotrf32Threads) {
    const int r = i >> 5, c = (i & 31) * 4;
    if (c > r) continue;
    const float4 v = *reinterpret_cast<const float4*>(As + r * kPLD + c);
    *reinterpret_cast<float4*>(S + base + (size_t)r * ld + c) =
        make_float4(v.x, c + 1 <= r ? v.y : 0.f, c + 2 <= r ? v.z : 0.f, c + 3 <= r ? v.w : 0.f);
    if ((c >> 5) <= (r >> 5))
      *reinterpret_cast<float4*>(Lout + (size_t)r * NB + c) = *reinterpret_cast<const float4*>(Xs + r * kPLD + c);
  }
}

}  // namespace nl
