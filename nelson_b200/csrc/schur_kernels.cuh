// schur_kernels.cuh -- reduced camera system S = U - W V^-1 W' and back-substitution.
//
// The algebra of SolverCholeskySchur::computeIncrement
// (nelson/SolverCholeskySchur.hpp:91-157), laid out the way
// SolverDiagonalBlocksInverseWWtMultSchur runs it
// (nelson/SolverDiagonalBlocksInverseWWtMultSchur.hpp:99-140):
//   vinv_kernel      MatrixDiagInv::compute (nelson/MatrixDiagInv.hpp:32-43):
//                    Vinv_p = inv(sym_upper(V_p) (1 + rel) + abs), register-resident
//                    3x3 LDL'.
//   wvinv_bs_kernel  MatrixWVinvMultiplier::multiply (MatrixWVinvMultiplier.hpp:33-35)
//                    Y = W Vinv per W block, and bS = -bU + Y bV per camera
//                    (= -bU - W xV0 of SolverCholeskySchur.hpp:114).
//   schur_kernel     MatrixWWtMultiplier::multiply (MatrixWWtMultiplier.hpp:139-152):
//                    S_ij = U_ij - sum_pairs Y_a W_b', one warp per output block over
//                    the block's pair list (no atomics), plus the diagonal damping of
//                    SolverCholeskySchur.hpp:121-124, written to dense lower storage.
//   backsub_kernel   MatrixWtXMultiplier::rightMultVectorSub + MatrixDiagInv::rightMultVector
//                    (MatrixWtXMultiplier.hpp:58-62, MatrixDiagInv.hpp:153-156):
//                    xV_p = Vinv_p (-bV_p - sum W' xU).
#pragma once

#include <type_traits>

#include "nl_common.cuh"

namespace nl {

struct SchurDev {
  int bc, nci, np, nU, nW, nS;
  int n, ld;                   // S size and leading dimension (n padded)
  const int* v_uid;            // point -> V uid (-1: none)
  const int* w_row_ptr;        // nci + 1 (CSR over internal cameras)
  const int* w_col;            // W uid -> point
  const int* w_row;            // W uid -> internal camera
  const int* w_col_ptr;        // np + 1 (CSC over points)
  const int* w_col_uid;        // W uids of a point, rows ascending
  const int* u_diag_uid;       // internal camera -> U uid of its diagonal block (-1: none)
  const int* s_i;              // output block -> block row i (i <= j)
  const int* s_j;              // output block -> block column j
  const int* s_uuid;           // output block -> U uid (-1: none)
  const long long* s_pair_ptr; // nS + 1
  const int* pair_a;           // W uid of (i, p)
  const int* pair_b;           // W uid of (j, p)
};

// ---------------------------------------------------------------------------
template <typename T, int BC>
static __global__ void vinv_kernel(SchurDev d, const T* __restrict__ V, T* __restrict__ Vinv, const double* __restrict__ lam,
                            int* __restrict__ status, const int* __restrict__ active) {
  constexpr int LV = Layout<T, BC>::V;
  if (active && !*active) return;
  const double rel = lam[0], abs = lam[1];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.np) return;
  const int q = d.v_uid[p];
  double a00 = 0, a01 = 0, a02 = 0, a11 = 0, a12 = 0, a22 = 0;
  if (q >= 0) {
    const T* v = V + (size_t)q * LV;
    a00 = v[0]; a01 = v[1]; a02 = v[2];
    a11 = v[4]; a12 = v[5]; a22 = v[8];
  }
  if (rel != 0.0 || abs != 0.0) {
    a00 = a00 * (1.0 + rel) + abs;
    a11 = a11 * (1.0 + rel) + abs;
    a22 = a22 * (1.0 + rel) + abs;
  }
  // LDL' of the symmetric 3x3 block (from its upper triangle)
  const double d0 = a00;
  const double l10 = a01 / d0, l20 = a02 / d0;
  const double d1 = a11 - l10 * a01;
  const double l21 = (a12 - l20 * a01) / d1;
  const double d2 = a22 - l20 * a02 - l21 * l21 * d1;
  const bool ok = d0 > 0.0 && d1 > 0.0 && d2 > 0.0 && isfinite(d0 + d1 + d2);
  if (!ok) atomicOr(status, ST_VINV_FAIL);
  // inv(L') D^-1 inv(L):  inv(L) = [[1,0,0],[-l10,1,0],[l10 l21 - l20, -l21, 1]]
  const double m10 = -l10, m21 = -l21, m20 = l10 * l21 - l20;
  const double i0 = 1.0 / d0, i1 = 1.0 / d1, i2 = 1.0 / d2;
  const double b00 = i0 + m10 * m10 * i1 + m20 * m20 * i2;
  const double b01 = m10 * i1 + m20 * m21 * i2;
  const double b02 = m20 * i2;
  const double b11 = i1 + m21 * m21 * i2;
  const double b12 = m21 * i2;
  const double b22 = i2;
  T* o = Vinv + (size_t)p * LV;
  o[0] = (T)b00; o[1] = (T)b01; o[2] = (T)b02;
  o[3] = (T)b01; o[4] = (T)b11; o[5] = (T)b12;
  o[6] = (T)b02; o[7] = (T)b12; o[8] = (T)b22;
}

// ---------------------------------------------------------------------------
template <typename T, int BC, int NT>
static __global__ void __launch_bounds__(NT) wvinv_bs_kernel(SchurDev d, const T* __restrict__ W,
                                                      const T* __restrict__ Vinv, T* __restrict__ Y,
                                                      const T* __restrict__ bU, const T* __restrict__ bV,
                                                      double* __restrict__ bS, const int* __restrict__ active) {
  constexpr int LW = Layout<T, BC>::W;
  constexpr int LV = Layout<T, BC>::V;
  __shared__ double red[NT / 32][BC];
  if (active && !*active) return;
  const int c = blockIdx.x;
  double acc[BC];
#pragma unroll
  for (int i = 0; i < BC; i++) acc[i] = 0.0;
  for (int q = d.w_row_ptr[c] + threadIdx.x; q < d.w_row_ptr[c + 1]; q += NT) {
    const int p = d.w_col[q];
    // blocks are padded to 16 bytes: move them as 16-byte vectors
    using V16 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    constexpr int EPV = 16 / (int)sizeof(T);
    __align__(16) T w[LW], v[LV], y[LW];
#pragma unroll
    for (int i = 0; i < LW / EPV; i++)
      reinterpret_cast<V16*>(w)[i] = __ldg(reinterpret_cast<const V16*>(W + (size_t)q * LW) + i);
#pragma unroll
    for (int i = 0; i < LV / EPV; i++)
      reinterpret_cast<V16*>(v)[i] = __ldg(reinterpret_cast<const V16*>(Vinv + (size_t)p * LV) + i);
    const T bv0 = bV[3 * (size_t)p], bv1 = bV[3 * (size_t)p + 1], bv2 = bV[3 * (size_t)p + 2];
#pragma unroll
    for (int i = 0; i < BC; i++) {
      const T w0 = w[i * 3], w1 = w[i * 3 + 1], w2 = w[i * 3 + 2];
      const T y0 = w0 * v[0] + w1 * v[3] + w2 * v[6];
      const T y1 = w0 * v[1] + w1 * v[4] + w2 * v[7];
      const T y2 = w0 * v[2] + w1 * v[5] + w2 * v[8];
      y[i * 3] = y0;
      y[i * 3 + 1] = y1;
      y[i * 3 + 2] = y2;
      acc[i] += (double)y0 * (double)bv0 + (double)y1 * (double)bv1 + (double)y2 * (double)bv2;
    }
#pragma unroll
    for (int i = BC * 3; i < LW; i++) y[i] = (T)0;
#pragma unroll
    for (int i = 0; i < LW / EPV; i++)
      reinterpret_cast<V16*>(Y + (size_t)q * LW)[i] = reinterpret_cast<const V16*>(y)[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < BC; i++) {
    const double v = warp_sum(acc[i]);
    if (lane == 0) red[warp][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < BC) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < NT / 32; w++) s += red[w][threadIdx.x];
    bS[(size_t)c * BC + threadIdx.x] = -(double)bU[(size_t)c * BC + threadIdx.x] + s;
  }
}

// ---------------------------------------------------------------------------
// One warp per output block (i <= j); lanes own the BC*BC outputs round-robin.
// Batches of PB pairs: lane l < 2 np loads one block UID (Y_a for l < np,
// W_b above), the operands move as 16-byte vectors (blocks are padded to 16
// bytes) and are re-laid in shared memory with rows padded to 4, so each
// 3-term row product reads two vectors.
template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
  using type = float4;
};
template <>
struct Vec4<double> {
  using type = double4;
};

// A staged row of a BC x 3 block (padded to 4 elements, 16-byte aligned).
__device__ __forceinline__ void load_row3(const float* p, float& a, float& b, float& c) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  a = v.x;
  b = v.y;
  c = v.z;
}
__device__ __forceinline__ void load_row3(const double* p, double& a, double& b, double& c) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  a = v.x;
  b = v.y;
  c = p[2];
}

// One warp per output block, blocks taken heaviest-first from a work counter
// (`order` lists them by pair count, descending), so the long diagonal blocks
// start early and the tail is short; each block is still summed by one warp
// in pair order, so S does not depend on the schedule.  Lane l < NSTR owns a
// 1 x SW strip (row r, columns c0 .. c0 + SW - 1) of the BC x BC block.
// Per batch of PB pairs the warp stages Y_a and W_b (rows padded to 4) in
// shared memory and already issues the global loads of the next batch, so
// their latency overlaps this batch's FMAs.  The batch's products are summed
// before they are subtracted (blocked summation: a diagonal block sums
// thousands of pairs in the working precision).
template <typename T, int BC, int WARPS>
static __global__ void __launch_bounds__(WARPS * 32, 2) schur_kernel(SchurDev d, const T* __restrict__ U,
                                                                      const T* __restrict__ Y, const T* __restrict__ W,
                                                                      const double* __restrict__ lam, T* __restrict__ S,
                                                                      T* __restrict__ S0, const int* __restrict__ order,
                                                                      int* __restrict__ counter,
                                                                      const int* __restrict__ active) {
  constexpr int LW = Layout<T, BC>::W;
  constexpr int LU = Layout<T, BC>::U;
  // pairs per batch: FP32 measured fastest at 10 (against 4, 6, 8, 12, 16 on
  // config 2); the FP64 comparison path keeps 8
  constexpr int PB = sizeof(T) == 4 ? 10 : 8;
  constexpr int SW = (BC % 3 == 0) ? 3 : ((BC % 2 == 0) ? 2 : 1);  // strip width
  constexpr int NSTR = BC * BC / SW;                               // strips (<= 32)
  constexpr int EPV = 16 / (int)sizeof(T);                         // elements per 16-byte vector
  constexpr int VB = LW / EPV;                                     // vectors per block
  constexpr int NV = (2 * PB * VB + 31) / 32;                      // staged vectors per lane
  using V16 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  static_assert(NSTR <= 32, "one strip per lane");
  __shared__ __align__(16) T sh[WARPS][2][PB][BC][4];
  if (active && !*active) return;
  const double rel = lam[0], abs = lam[1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = lane / (BC / SW), c0 = (lane % (BC / SW)) * SW;
  const bool own = lane < NSTR;
  T(*sy)[BC][4] = sh[warp][0];
  T(*sw)[BC][4] = sh[warp][1];
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(counter, 1);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= d.nS) break;
    const int b = order[idx];
    const int bi = d.s_i[b], bj = d.s_j[b], uu = d.s_uuid[b];
    T acc[SW];
#pragma unroll
    for (int s2 = 0; s2 < SW; s2++)
      acc[s2] = (own && uu >= 0) ? U[(size_t)uu * LU + r * BC + c0 + s2] : (T)0;
    const long long p0 = d.s_pair_ptr[b], p1 = d.s_pair_ptr[b + 1];
    // batch loader: lanes 0..np-1 fetch pair_a, np..2np-1 pair_b, then the
    // 2 np blocks are read as VB 16-byte vectors each
    V16 v[NV];
    int np = 0;
    auto load_batch = [&](long long pp) {
      np = (int)min((long long)PB, p1 - pp);
      int uid = 0;
      if (lane < np) uid = __ldg(d.pair_a + pp + lane);
      else if (lane < 2 * np) uid = __ldg(d.pair_b + pp + lane - np);
#pragma unroll
      for (int t = 0; t < NV; t++) {
        const int u = lane + 32 * t;
        const int blk = u / VB, part = u - blk * VB;
        const int src_uid = __shfl_sync(0xffffffffu, uid, blk & 31);
        if (blk < 2 * np) {
          const T* base = (blk < np ? Y : W) + (size_t)src_uid * LW;
          v[t] = __ldg(reinterpret_cast<const V16*>(base + part * EPV));
        }
      }
    };
    if (p0 < p1) load_batch(p0);
    for (long long pp = p0; pp < p1; pp += PB) {
      const int cur = np;
      // registers -> shared memory (rows padded to 4)
#pragma unroll
      for (int t = 0; t < NV; t++) {
        const int u = lane + 32 * t;
        const int blk = u / VB, part = u - blk * VB;
        if (blk < 2 * cur) {
          T(*dst)[4] = blk < cur ? sy[blk] : sw[blk - cur];
          const T* e = reinterpret_cast<const T*>(&v[t]);
#pragma unroll
          for (int m = 0; m < EPV; m++) {
            const int el = part * EPV + m;  // element of the BC x 3 block
            if (el < BC * 3) dst[el / 3][el % 3] = e[m];
          }
        }
      }
      __syncwarp();
      if (pp + PB < p1) load_batch(pp + PB);  // in flight during the FMAs below
      if (own) {
        T part[SW];
#pragma unroll
        for (int s2 = 0; s2 < SW; s2++) part[s2] = (T)0;
        for (int q = 0; q < cur; q++) {
          T y0, y1, y2;
          load_row3(sy[q][r], y0, y1, y2);
#pragma unroll
          for (int s2 = 0; s2 < SW; s2++) {
            T w0, w1, w2;
            load_row3(sw[q][c0 + s2], w0, w1, w2);
            part[s2] += y0 * w0 + y1 * w1 + y2 * w2;
          }
        }
#pragma unroll
        for (int s2 = 0; s2 < SW; s2++) acc[s2] -= part[s2];
      }
      __syncwarp();
    }
    // damping on the diagonal of diagonal blocks, then the store (lower storage:
    // S_lower[j*BC + c][i*BC + r] = S_ij[r][c])
    if (own) {
      const int ud = (bi == bj) ? d.u_diag_uid[bi] : -1;
#pragma unroll
      for (int s2 = 0; s2 < SW; s2++) {
        const int cc = c0 + s2;
        T val = acc[s2];
        if (bi == bj && r == cc && (rel != 0.0 || abs != 0.0)) {
          const double udg = ud >= 0 ? (double)U[(size_t)ud * LU + r * BC + r] : 0.0;
          val = (T)((double)val + rel * udg + abs);
        }
        const size_t o = (size_t)(bj * BC + cc) * d.ld + (size_t)(bi * BC + r);
        if (bi != bj || cc >= r) {
          S[o] = val;
          if (S0) S0[o] = val;
        }
      }
    }
  }
}

// Zero the tiles of S (and S0) that can hold nonzeros: row r of tile row I
// over columns [env_first[I] NB, (I + 1) NB) -- the Cholesky envelope.  The
// other tiles are zero after the first full clear and stay exactly zero: the
// Schur blocks lie inside the envelope, and the factorisation writes only
// zeros there (TRSM and trailing updates of zero tiles).  One CTA per row.
template <typename T>
static __global__ void clear_envelope_kernel(T* __restrict__ S, T* __restrict__ S0, int ld, int nb,
                                             const int* __restrict__ env_first, const int* __restrict__ active) {
  if (active && !*active) return;
  const int r = blockIdx.x, I = r / nb;
  const size_t c0 = (size_t)env_first[I] * nb, c1 = (size_t)(I + 1) * nb;
  constexpr int EPV = 16 / (int)sizeof(T);  // elements per 16-byte store
  using V16 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  const V16 z = {};
  for (size_t c = c0 + (size_t)threadIdx.x * EPV; c < c1; c += (size_t)blockDim.x * EPV) {
    *reinterpret_cast<V16*>(S + (size_t)r * ld + c) = z;
    if (S0) *reinterpret_cast<V16*>(S0 + (size_t)r * ld + c) = z;
  }
}

// Identity on the padded tail of S (rows n .. ld-1).
template <typename T>
static __global__ void pad_identity_kernel(T* __restrict__ S, T* __restrict__ S0, int n, int ld,
                                    const int* __restrict__ active) {
  if (active && !*active) return;
  const int i = n + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ld) return;
  S[(size_t)i * ld + i] = (T)1;
  if (S0) S0[(size_t)i * ld + i] = (T)1;
}

// ---------------------------------------------------------------------------
template <typename T, int BC>
static __global__ void backsub_kernel(SchurDev d, const T* __restrict__ W, const T* __restrict__ Vinv,
                               const T* __restrict__ bV, const double* __restrict__ xU, double* __restrict__ xV,
                               const int* __restrict__ ok_flag, const int* __restrict__ active) {
  constexpr int LW = Layout<T, BC>::W;
  constexpr int LV = Layout<T, BC>::V;
  if (active && !*active) return;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.np) return;
  if (ok_flag && *ok_flag != 0) {  // failed factorisation: zero increment
    xV[3 * (size_t)p] = 0.0;
    xV[3 * (size_t)p + 1] = 0.0;
    xV[3 * (size_t)p + 2] = 0.0;
    return;
  }
  double t0 = -(double)bV[3 * (size_t)p], t1 = -(double)bV[3 * (size_t)p + 1], t2 = -(double)bV[3 * (size_t)p + 2];
  for (int s = d.w_col_ptr[p]; s < d.w_col_ptr[p + 1]; s++) {
    const int q = d.w_col_uid[s];
    const int c = d.w_row[q];
    using V16 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    constexpr int EPV = 16 / (int)sizeof(T);
    __align__(16) T w[LW];
#pragma unroll
    for (int i = 0; i < LW / EPV; i++)
      reinterpret_cast<V16*>(w)[i] = __ldg(reinterpret_cast<const V16*>(W + (size_t)q * LW) + i);
    const double* x = xU + (size_t)c * BC;
#pragma unroll
    for (int i = 0; i < BC; i++) {
      const double xi = x[i];
      t0 -= (double)w[i * 3] * xi;
      t1 -= (double)w[i * 3 + 1] * xi;
      t2 -= (double)w[i * 3 + 2] * xi;
    }
  }
  const T* v = Vinv + (size_t)p * LV;
  xV[3 * (size_t)p] = (double)v[0] * t0 + (double)v[1] * t1 + (double)v[2] * t2;
  xV[3 * (size_t)p + 1] = (double)v[3] * t0 + (double)v[4] * t1 + (double)v[5] * t2;
  xV[3 * (size_t)p + 2] = (double)v[6] * t0 + (double)v[7] * t1 + (double)v[8] * t2;
}

}  // namespace nl
