// cholesky.cuh -- blocked right-looking Cholesky of the reduced camera system.
//
// Replaces the dense LDLT factorisation + solve of SolverCholeskySchur
// (SolverCholeskyEigenDense::factorize/solve, nelson/SolverCholeskyDense.hpp:15-24,
// used at nelson/SolverCholeskySchur.hpp:136-140).  S is stored dense,
// row-major, lower triangle, n padded to a multiple of NB = 128 (identity on
// the padding).  Per 128-wide panel k:
//   potrf_diag_kernel  factor of the diagonal tile and its inverse (one CTA)
//   trsm_kernel        L_ik = A_ik L_kk^-T as a product with the inverse
//   syrk update        A_ij -= L_ik L_jk' on the trailing lower triangle
//                      (tensor-core kernel in tc_syrk.cu for the mixed path,
//                      cuBLAS DSYRK for the FP64 comparison path)
// Solves use the tile inverses: trsv_fwd/bwd_kernel with a ticketed
// look-back between CTAs of one launch, each wait bounded.
#pragma once

#include "nl_common.cuh"
#include "tc_pack_layout.cuh"

namespace nl {

constexpr int NB = 128;
constexpr long long kSpinLimit = 1LL << 24;  // default bound of the flag waits (~1 s worst case)

// Programmatic dependent launch of the critical-path chain (potrf -> row-tile
// TRSM -> diagonal-tile update -> potrf ...): each kernel lets the next one in
// its stream launch at its start, and waits for its predecessor's completion
// (and memory flush) before touching what that predecessor wrote.  Both are
// no-ops for a kernel launched without the attribute.
__device__ inline void chain_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ inline void chain_release() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// One CTA: factor the NB x NB diagonal tile of panel k in the storage
// precision T (FP64 for the FP64 path; FP32 for the mixed path, whose
// trailing updates and off-diagonal solves are FP32-accurate as well and whose
// factor only preconditions the FP64 refinement) and build its inverse, in
// registers, as 32 super-steps of 4 columns.
//
// Owner threads (528): thread t owns 4x4 block (R, C), C <= R, of the lower
// triangle and one register block for it: A until block column C is factored,
// afterwards B -> X = inv(L) (right-looking forward substitution of L X = I).
// Pivot warp (warp 14): does all per-super-step work that is not a bulk update,
// so that no owner warp runs it for one or two active lanes.  Super-step jb:
//   (2) pivot warp, lane l < 31: for the row-jb block (jb, C = l) if l < jb,
//       else for the column-jb block (R = l + 1, jb): out = M Di' with M the
//       staged B' (row block: X_jb,C = out') or A (column block: L_R,jb =
//       out); publishes L / X in shared memory and writes them to S / Linv.
//   (3) owners with jb < R (except the next diagonal block) apply one rank-4
//       update  t -= L_R,jb Q_jb,C  with Q = L_C,jb' while jb < C (A part) and
//       Q = X_jb,C once jb >= C (X part) -- the same instructions for both --
//       then stage their block in shared memory if it just became final:
//       column-(jb+1) blocks (A), row-(jb+1) blocks (B'), diagonal block jb+2.
//       Concurrently the pivot warp's lane jb, which holds L_jb+1,jb, factors
//       the next diagonal block A_jb+1,jb+1 - L_jb+1,jb L_jb+1,jb' and inverts
//       it (Di of super-step jb+1): the serial 4x4 factor overlaps the updates.
// Warps are spread over the SM's four schedulers by index mod 4; the pivot
// warp's scheduler carries three owner warps, the others four or five.
// Shared 4x4 blocks are 20-word rows (16 used): lanes reading or writing
// consecutive blocks with 16-byte vectors stay within the minimum wavefronts.
// Two barriers per super-step.  L_kk is written to S and the blocks of
// inv(L_kk) on and below the diagonal to Linv (its strictly upper blocks are
// never written: the caller keeps them zero).
constexpr int kPivotWarp = 14;
constexpr int PT = 32 * 18;  // 17 owner warps (528 owners) + the pivot warp
constexpr int kTiles4 = (NB / 4) * (NB / 4 + 1) / 2;  // 528
constexpr int kBlk = 20;     // words per shared 4x4 block
constexpr size_t kPotrfSmem = 0;

// four consecutive elements (16-byte aligned for float, 32 for double; any
// address space)
__device__ inline void store_row4(float* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
__device__ inline void store_row4(double* p, double a, double b, double c, double d) {
  reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
  reinterpret_cast<double2*>(p)[1] = make_double2(c, d);
}
__device__ inline void load_row4(const float* p, float v[4]) {
  const float4 x = *reinterpret_cast<const float4*>(p);
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ inline void load_row4(const double* p, double v[4]) {
  const double2 x = reinterpret_cast<const double2*>(p)[0], y = reinterpret_cast<const double2*>(p)[1];
  v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}

// 1 / sqrt of a pivot, clamped away from zero (a non-positive pivot is
// flagged separately)
__device__ inline float pivot_rsqrt(float d) { return rsqrtf(fmaxf(d, 1e-30f)); }
__device__ inline double pivot_rsqrt(double d) { return rsqrt(fmax(d, 1e-300)); }

// Factor the 4x4 SPD block a (lower part used) of diagonal block jb and invert
// the factor: L to S (zeros above its diagonal), Di = inv(L) to the shared Di
// (row-major 4x4) and X block (row i, column c at i * 4 + c) and to Linv.
// Returns false on a non-positive pivot.
template <typename T>
__device__ inline bool factor_pivot_block(T a[4][4], int jb, T* __restrict__ S, size_t base, int ld,
                                          T* __restrict__ Lout, T* Di, T* Xblk) {
  bool fail = false;
  T rs[4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    T d = a[j][j];
#pragma unroll
    for (int l = 0; l < j; l++) d -= a[j][l] * a[j][l];
    fail |= !(d > (T)0) || !isfinite(d);
    rs[j] = pivot_rsqrt(d);
    a[j][j] = d * rs[j];
#pragma unroll
    for (int i = j + 1; i < 4; i++) {
      T v = a[i][j];
#pragma unroll
      for (int l = 0; l < j; l++) v -= a[i][l] * a[j][l];
      a[i][j] = v * rs[j];
    }
  }
  const int r0 = 4 * jb;
#pragma unroll
  for (int i = 0; i < 4; i++)
    store_row4(S + base + (size_t)(r0 + i) * ld + r0, a[i][0], i >= 1 ? a[i][1] : (T)0, i >= 2 ? a[i][2] : (T)0,
               i >= 3 ? a[i][3] : (T)0);
  // inv(L) one column at a time: multiplications only (the rsqrt is 1 / L_ii)
  T di[4][4];
#pragma unroll
  for (int c = 0; c < 4; c++)
#pragma unroll
    for (int i = 0; i < 4; i++) {
      if (i < c) {
        di[i][c] = (T)0;
      } else if (i == c) {
        di[i][c] = rs[i];
      } else {
        T v = (T)0;
#pragma unroll
        for (int l = c; l < i; l++) v -= a[i][l] * di[l][c];
        di[i][c] = v * rs[i];
      }
    }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    store_row4(Di + 4 * i, di[i][0], di[i][1], di[i][2], di[i][3]);
    store_row4(Xblk + 4 * i, di[i][0], di[i][1], di[i][2], di[i][3]);
    store_row4(Lout + (size_t)(r0 + i) * NB + r0, di[i][0], di[i][1], di[i][2], di[i][3]);
  }
  return !fail;
}

template <typename T>
static __global__ void __launch_bounds__(PT) potrf_diag_kernel(T* __restrict__ S, int ld, int k,
                                                               T* __restrict__ Linv, int* __restrict__ status,
                                                               const int* __restrict__ active) {
  // Published blocks of super-step jb (double-buffered): L_R,jb at Lc[.][R]
  // (row u, column w at w * 4 + u) and X_jb,C at Xr[.][C] (row w, column v at
  // w * 4 + v), so that rank-4 step w reads 4 consecutive words of each.
  // Staged blocks M at Mst[slot] (row u, column w at u * 4 + w; row block C:
  // slot C, holding B'; column block R: slot R - 1, holding A); staged
  // diagonal blocks by parity.
  __shared__ __align__(16) T Lc[2][NB / 4][kBlk];
  __shared__ __align__(16) T Xr[2][NB / 4][kBlk];
  __shared__ __align__(16) T Mst[NB / 4][kBlk];
  __shared__ __align__(16) T Di[2][16];  // inv(L_jb,jb), row-major
  __shared__ T Dst[2][4][4];
  __shared__ int bad;
  chain_release();
  chain_wait();
  if (active && !*active) return;
  const int tid = threadIdx.x, lane = tid & 31, wi = tid >> 5;
  const bool pivot = wi == kPivotWarp;
  const int oid = wi < kPivotWarp ? tid : tid - 32;  // owner index
  const size_t base = (size_t)k * NB * ld + (size_t)k * NB;
  T* Lout = Linv + (size_t)k * NB * NB;
  if (tid == 0) bad = 0;
  int R = 0, C = 0;
  const bool own = !pivot && oid < kTiles4;
  if (own) {
    R = (int)((sqrtf(8.0f * oid + 1.0f) - 1.0f) * 0.5f);
    while ((R + 1) * (R + 2) / 2 <= oid) R++;
    while (R * (R + 1) / 2 > oid) R--;
    C = oid - R * (R + 1) / 2;
  }
  const int r0 = 4 * R, c0 = 4 * C;
  T t[4][4];
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++)
      t[u][v] = (own && c0 + v <= r0 + u) ? S[base + (size_t)(r0 + u) * ld + c0 + v] : (T)0;
  // stage column 0 and the first two diagonal blocks
  if (own && C == 0 && R > 0) {
#pragma unroll
    for (int u = 0; u < 4; u++) {
      store_row4(&Mst[R - 1][4 * u], t[u][0], t[u][1], t[u][2], t[u][3]);
#pragma unroll
      for (int w = 0; w < 4; w++) t[u][w] = (T)0;
    }
  } else if (own && R == C && R <= 1) {
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int v = 0; v < 4; v++) Dst[R][u][v] = t[u][v];
  }
  __syncthreads();
  if (pivot && lane == 0) {
    T a[4][4];
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int v = 0; v < 4; v++) a[u][v] = Dst[0][u][v];
    if (!factor_pivot_block(a, 0, S, base, ld, Lout, Di[0], Xr[0][0])) bad = 1;
  }
  __syncthreads();
  T out[4][4];  // pivot warp: this super-step's L (or X') block
  for (int jb = 0; jb < NB / 4; jb++) {
    const int buf = jb & 1;
    // (2) the row-jb and column-jb blocks, one per pivot-warp lane
    if (pivot && lane < NB / 4 - 1) {
      T m[4][4], d[4][4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        load_row4(&Mst[lane][4 * u], m[u]);
        load_row4(&Di[buf][4 * u], d[u]);
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          T s = (T)0;
#pragma unroll
          for (int w = 0; w <= v; w++) s += m[u][w] * d[v][w];
          out[u][v] = s;
        }
      const bool rowb = lane < jb;
      const int idx = rowb ? lane : lane + 1;  // C of a row block, R of a column block
      // L_R,jb[u][v] at v * 4 + u; X_jb,C[v][u] = out[u][v] at v * 4 + u
      T* pub = rowb ? Xr[buf][idx] : Lc[buf][idx];
#pragma unroll
      for (int v = 0; v < 4; v++) store_row4(pub + 4 * v, out[0][v], out[1][v], out[2][v], out[3][v]);
      if (rowb) {
        // X_jb,C = out': row v of X is column v of out
#pragma unroll
        for (int v = 0; v < 4; v++)
          store_row4(Lout + (size_t)(4 * jb + v) * NB + 4 * idx, out[0][v], out[1][v], out[2][v], out[3][v]);
      } else {
#pragma unroll
        for (int u = 0; u < 4; u++)
          store_row4(S + base + (size_t)(4 * idx + u) * ld + 4 * jb, out[u][0], out[u][1], out[u][2], out[u][3]);
      }
    }
    __syncthreads();
    // (3) one rank-4 update per block below row jb, then staging; the next
    //     step writes the other buffers, so no barrier here
    if (own && jb < R && !(R == C && R == jb + 1)) {
      const T* q = (jb < C) ? Lc[buf][C] : Xr[buf][C];  // Q_jb,C row w at 4 w either way
#pragma unroll
      for (int w = 0; w < 4; w++) {
        T pr[4], qc[4];
        load_row4(&Lc[buf][R][4 * w], pr);
        load_row4(q + 4 * w, qc);
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
          for (int v = 0; v < 4; v++) t[u][v] -= pr[u] * qc[v];
      }
      if (C == jb + 1 && R > jb + 1) {  // A_R,jb+1 is final
#pragma unroll
        for (int u = 0; u < 4; u++) {
          store_row4(&Mst[R - 1][4 * u], t[u][0], t[u][1], t[u][2], t[u][3]);
#pragma unroll
          for (int w = 0; w < 4; w++) t[u][w] = (T)0;  // the X block starts from zero below the diagonal
        }
      } else if (R == jb + 1) {  // B_jb+1,C is final (C <= jb): stage B'
#pragma unroll
        for (int u = 0; u < 4; u++) store_row4(&Mst[C][4 * u], t[0][u], t[1][u], t[2][u], t[3][u]);
      } else if (R == C && R == jb + 2) {  // all but the last update of A_jb+2,jb+2
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
          for (int v = 0; v < 4; v++) Dst[R & 1][u][v] = t[u][v];
      }
    }
    // look-ahead: the next diagonal block, from its staged value and the
    // L_jb+1,jb held by lane jb
    if (pivot && lane == jb && jb + 1 < NB / 4) {
      const int nb = jb + 1;
      T a[4][4];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int c = 0; c <= i; c++) {
          T v = Dst[nb & 1][i][c];
#pragma unroll
          for (int w = 0; w < 4; w++) v -= out[i][w] * out[c][w];
          a[i][c] = v;
        }
      if (!factor_pivot_block(a, nb, S, base, ld, Lout, Di[nb & 1], Xr[nb & 1][nb])) bad = 1;
    }
    __syncthreads();
  }
  if (tid == 0 && bad) atomicOr(status, ST_CHOL_FAIL);
}

// ---------------------------------------------------------------------------
// L_ik = A_ik inv(L_kk)' for 64-row slabs of rows [row_begin, row_begin +
// nrows) below the diagonal tile (absolute row indices), as a
// register-tiled product: X (64 x 128) = A (64 x 128) Linv' (128 x 128).
// 256 threads, thread (ty, tx) computes rows ty*4 .. ty*4+3 (ty < 16) and
// columns tx + 16 j (tx < 16, j < 8); A and Linv are staged in shared memory
// in the working precision, K-major, and read as broadcasts / strided rows.
constexpr int TRSM_ROWS = 64;
template <typename T>
constexpr size_t trsm_smem() {
  return sizeof(T) * ((size_t)NB * (NB + 1) + (size_t)NB * (TRSM_ROWS + 1));
}

template <typename T>
static __global__ void __launch_bounds__(256) trsm_kernel(T* __restrict__ S, int ld, int k, int row_begin, int nrows,
                                                          const T* __restrict__ Linv,
                                                          uint8_t* __restrict__ pack,
                                                          const int* __restrict__ active) {
  extern __shared__ unsigned char smraw[];
  T* sL = reinterpret_cast<T*>(smraw);      // sL[l][j] = Linv[j][l], (NB + 1) stride
  T* sA = sL + NB * (NB + 1);               // sA[l][r] = A[r][l], (TRSM_ROWS + 1) stride
  if (active && !*active) return;
  const int tid = threadIdx.x;
  const int r0 = row_begin + blockIdx.x * TRSM_ROWS;
  const int nr = min(TRSM_ROWS, row_begin + nrows - r0);
  if (nr <= 0) return;
  // staging: 16 independent loads in flight per thread before the stores
  const T* Li = Linv + (size_t)k * NB * NB;
#pragma unroll 1
  for (int i0 = tid; i0 < NB * NB; i0 += 256 * 16) {
    T v[16];
#pragma unroll
    for (int u = 0; u < 16; u++) v[u] = __ldg(Li + i0 + 256 * u);
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int i = i0 + 256 * u, j = i / NB, l = i - j * NB;
      sL[l * (NB + 1) + j] = v[u];
    }
  }
#pragma unroll 1
  for (int i0 = tid; i0 < TRSM_ROWS * NB; i0 += 256 * 16) {
    T v[16];
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int i = i0 + 256 * u, r = i / NB, l = i - r * NB;
      v[u] = r < nr ? S[(size_t)(r0 + r) * ld + (size_t)k * NB + l] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < 16; u++) {
      const int i = i0 + 256 * u, r = i / NB, l = i - r * NB;
      sA[l * (TRSM_ROWS + 1) + r] = v[u];
    }
  }
  __syncthreads();
  const int ty = tid >> 4, tx = tid & 15;
  T acc[4][8];
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 8; v++) acc[u][v] = (T)0;
#pragma unroll 4
  for (int l = 0; l < NB; l++) {
    T a[4], b[8];
#pragma unroll
    for (int u = 0; u < 4; u++) a[u] = sA[l * (TRSM_ROWS + 1) + ty * 4 + u];
#pragma unroll
    for (int v = 0; v < 8; v++) b[v] = sL[l * (NB + 1) + tx + 16 * v];
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int v = 0; v < 8; v++) acc[u][v] += a[u] * b[v];
  }
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int rr = ty * 4 + u;
    if (rr < nr) {
#pragma unroll
      for (int v = 0; v < 8; v++) S[(size_t)(r0 + rr) * ld + (size_t)k * NB + tx + 16 * v] = acc[u][v];
    }
  }
  if (sizeof(T) == 4 && pack) {
    // BF16 hi/lo pack of this slab for the tensor-core update: stage it
    // row-major over the operand buffer (64 x 130 floats fit in sA), then
    // each item is 8 consecutive columns of one row
    constexpr int kSt = NB + 2;
    static_assert(TRSM_ROWS * kSt <= NB * (TRSM_ROWS + 1), "staging fits the operand buffer");
    float* st = reinterpret_cast<float*>(sA);
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int v = 0; v < 8; v++) st[(ty * 4 + u) * kSt + tx + 16 * v] = (float)acc[u][v];
    __syncthreads();
    const int rel0 = r0 - (k + 1) * NB;  // pack rows start below the diagonal tile
    for (int i = tid; i < TRSM_ROWS * 16; i += 256) {
      const int rr = i >> 4, h = i & 15;
      if (rr >= nr) continue;
      float x[8];
#pragma unroll
      for (int q = 0; q < 8; q++) x[q] = st[rr * kSt + 8 * h + q];
      tc_pack_store8(pack, tc_pack_offset(rel0 + rr, h), x);
    }
  }
}

// ---------------------------------------------------------------------------
// Critical-path kernels of the tensor-core schedule (FP32).  Each runs as
// 128 / RPC CTAs of 256 threads, CTA c owning an RPC-row slice of one
// 128 x 128 tile (RPC = kChainRows below):
//   trsm_tile_kernel    L_(j+1),j = A_(j+1),j inv(L_jj)' for row tile j+1 of
//                       panel j, and its BF16 pack
//   diag_update_kernel  A_tt -= sum_p L_t,p L_t,p' on diagonal tile t over
//                       panels p in [p0, p0 + np)
// Thread (w, lane) of an RPC x 128 slice computes RPC / 2 row pairs (the
// lane's pair lane / CG, CG = 64 / RPC) and columns 16 w + lane % CG + CG m
// (m < 16 / CG).  Both operands stay row-major in shared memory (row stride
// 132 floats) and are read as float4 along K.
constexpr int kSliceRows = 16;  // rows per CTA of the chain kernels at most (shared-memory sizes)
// Rows per CTA of the row-tile TRSM and the diagonal-tile update on the
// factorisation's critical path: 4 (32 CTAs).  Config 2, LM it/s on the
// B200 with identical results: 16 rows (8 CTAs) 93.1, 8 rows 94.6, 4 rows
// 95.6 -- every CTA stages the whole panel, so more CTAs cut each one's
// FMAs, not its copies.
constexpr int kChainRows = 4;
static_assert(kChainRows == 16 || kChainRows == 8 || kChainRows == 4, "chain kernels: 4, 8 or 16 rows per CTA");
constexpr int kSlLd = NB + 4;                // 132
constexpr size_t kTrsmTileSmem = sizeof(float) * (size_t)(NB + kSliceRows) * kSlLd;  // 76,032 B
constexpr size_t kDiagUpdSmem = sizeof(float) * (size_t)NB * kSlLd;                 // 67,584 B per panel

// acc[h][m] += sum_l a_h[l] b[16 w + (lane & 3) + 4 m][l], l < NB
// A CTA of the chain kernels owns RPC rows of a 128 x 128 result as RPC / 2
// row pairs (a0, a1); warp w owns columns 16 w .. 16 w + 15.  Lane l: pair
// l / CG, columns 16 w + l % CG + CG m (m < 16 / CG), CG = 32 / (RPC / 2).
// Each output sums over l = 0 .. 127 in order (x, y, z, w of every float4).
template <int RPC>
__device__ inline void slice_mma(const float* __restrict__ a0, const float* __restrict__ a1,
                                 const float* __restrict__ sb, int lane, int w, float acc[2][16 / (64 / RPC)]) {
  constexpr int CG = 64 / RPC, M = 16 / CG;
  const float* pb = sb + (16 * w + (lane % CG)) * kSlLd;
#pragma unroll 4
  for (int l = 0; l < NB; l += 4) {
    float4 a[2], b[M];
    a[0] = *reinterpret_cast<const float4*>(a0 + l);
    a[1] = *reinterpret_cast<const float4*>(a1 + l);
#pragma unroll
    for (int m = 0; m < M; m++) b[m] = *reinterpret_cast<const float4*>(pb + CG * m * kSlLd + l);
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int m = 0; m < M; m++) {
        acc[h][m] = fmaf(a[h].x, b[m].x, acc[h][m]);
        acc[h][m] = fmaf(a[h].y, b[m].y, acc[h][m]);
        acc[h][m] = fmaf(a[h].z, b[m].z, acc[h][m]);
        acc[h][m] = fmaf(a[h].w, b[m].w, acc[h][m]);
      }
  }
}

// 16-byte global -> shared copies that complete asynchronously: a kernel
// issues all of its staging before one wait, so the staging costs one L2 /
// HBM round trip however loaded the memory system is
__device__ inline void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ inline void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// rows x 128 FP32 columns (row stride ld) into shared memory (stride kSlLd)
__device__ inline void stage_rows_f32(const float* __restrict__ src, size_t ld, int rows, float* __restrict__ dst,
                                      int tid) {
  for (int e = tid; e < rows * NB / 4; e += 256) {
    const int r = e >> 5, c4 = e & 31;
    cp_async16(dst + r * kSlLd + 4 * c4, src + (size_t)r * ld + 4 * c4);
  }
}

template <int RPC>
static __global__ void __launch_bounds__(256) trsm_tile_kernel(float* __restrict__ S, int ld, int j,
                                                               const float* __restrict__ Linv,
                                                               uint8_t* __restrict__ pack,
                                                               const int* __restrict__ active) {
  constexpr int P = RPC / 2, CG = 32 / P, M = 16 / CG;
  extern __shared__ float4 smf4[];
  float* sb = reinterpret_cast<float*>(smf4);  // inv(L_jj), row i = output column i
  float* sa = sb + NB * kSlLd;                 // the slice's RPC rows of A_(j+1),j
  chain_release();
  chain_wait();
  if (active && !*active) return;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int rel0 = blockIdx.x * RPC;  // first slice row within the tile
  float* A = S + (size_t)((j + 1) * NB + rel0) * ld + (size_t)j * NB;
  stage_rows_f32(Linv + (size_t)j * NB * NB, NB, NB, sb, tid);  // zeros above the diagonal included
  stage_rows_f32(A, ld, RPC, sa, tid);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  float acc[2][M] = {};
  const float* a0 = sa + (lane / CG) * kSlLd;
  slice_mma<RPC>(a0, a0 + P * kSlLd, sb, lane, w, acc);
  // stage the slice of L row-major over the A rows, then store rows to S
  // (float4) and the pack (8 consecutive columns per item)
  __syncthreads();
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int m = 0; m < M; m++) sa[((lane / CG) + P * h) * kSlLd + 16 * w + (lane % CG) + CG * m] = acc[h][m];
  __syncthreads();
  for (int e = tid; e < RPC * NB / 4; e += 256) {
    const int r = e >> 5, c4 = e & 31;
    *reinterpret_cast<float4*>(A + (size_t)r * ld + 4 * c4) = *reinterpret_cast<const float4*>(sa + r * kSlLd + 4 * c4);
  }
  if (pack) {
    for (int e = tid; e < RPC * 16; e += 256) {
      const int r = e >> 4, h = e & 15;
      float x[8];
#pragma unroll
      for (int q = 0; q < 8; q++) x[q] = sa[r * kSlLd + 8 * h + q];
      tc_pack_store8(pack, tc_pack_offset(rel0 + r, h), x);
    }
  }
}

// Slice c of RPC rows owns tile rows P c .. P c + P - 1 and 127 - P c - P + 1
// .. 127 - P c (P = RPC / 2): equal shares of the lower triangle.  A_tt's
// lower triangle only is written.  np <= 4 panels through two staging
// buffers (min(np, 2) x kDiagUpdSmem bytes of shared memory): panel p + 2 is
// copied in while panel p + 1 is applied.
constexpr int kDiagUpdMaxPanels = 4;
template <int RPC>
__device__ inline int diag_slice_row(int c, int p) {
  constexpr int P = RPC / 2;
  return p < P ? P * c + p : NB - 1 - P * c - (p - P);
}

template <int RPC>
static __global__ void __launch_bounds__(256) diag_update_kernel(float* __restrict__ S, int ld, int t, int p0, int np,
                                                                 const int* __restrict__ active) {
  constexpr int P = RPC / 2, CG = 32 / P, M = 16 / CG;
  extern __shared__ float4 smf4[];
  float* sm = reinterpret_cast<float*>(smf4);  // L_t,p (all 128 rows) per panel
  chain_release();
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, c = blockIdx.x;
  const int ra = diag_slice_row<RPC>(c, lane / CG), rb = diag_slice_row<RPC>(c, P + lane / CG);
  const float* T0 = S + (size_t)t * NB * ld + (size_t)p0 * NB;
  // all panels but the last were finished before the stream's preceding
  // kernel (the row-tile TRSM of the last one) started: fetch the first while
  // that kernel runs
  if (np > 1) stage_rows_f32(T0, ld, NB, sm, tid);
  cp_async_commit();
  chain_wait();
  if (active && !*active) {
    cp_async_wait<0>();
    return;
  }
  if (np > 1)
    stage_rows_f32(T0 + NB, ld, NB, sm + NB * kSlLd, tid);
  else
    stage_rows_f32(T0, ld, NB, sm, tid);
  cp_async_commit();
  float acc[2][M] = {};
  for (int p = 0; p < np; p++) {
    // committed groups so far: panels 0 .. min(p + 1, np - 1) (one empty
    // group when np == 1); panel p is complete once at most the newest is
    // still in flight
    if (p + 1 < np)
      cp_async_wait<1>();
    else
      cp_async_wait<0>();
    __syncthreads();
    const float* sb = sm + (p & 1) * NB * kSlLd;
    slice_mma<RPC>(sb + ra * kSlLd, sb + rb * kSlLd, sb, lane, w, acc);
    __syncthreads();  // every warp is done with buffer p & 1
    if (p + 2 < np) {
      stage_rows_f32(T0 + (size_t)(p + 2) * NB, ld, NB, sm + (p & 1) * NB * kSlLd, tid);
      cp_async_commit();
    }
  }
  float* D = S + (size_t)t * NB * ld + (size_t)t * NB;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int r = h ? rb : ra;
#pragma unroll
    for (int m = 0; m < M; m++) {
      const int i = 16 * w + (lane % CG) + CG * m;
      if (i <= r) D[(size_t)r * ld + i] -= acc[h][m];
    }
  }
}

// ---------------------------------------------------------------------------
// CUDA-core trailing update (FP32 or FP64), one CTA per 128 x 128 lower tile:
// C_IJ -= X_I X_J' with X = columns [k NB, (k+1) NB).  Used as the portable
// reference of the tensor-core kernel and for small problems.
template <typename T>
__device__ inline void syrk_cc_tile(T* __restrict__ S, int ld, int k, int gI, int gJ);

template <typename T>
static __global__ void __launch_bounds__(256) syrk_cc_kernel(T* __restrict__ S, int ld, int k, int t0, int nt,
                                                      const int* __restrict__ active) {
  if (active && !*active) return;
  const int q = blockIdx.x;
  int I = (int)((sqrt(8.0 * q + 1.0) - 1.0) * 0.5);
  while ((I + 1) * (I + 2) / 2 <= q) I++;
  while (I * (I + 1) / 2 > q) I--;
  const int J = q - I * (I + 1) / 2;
  syrk_cc_tile<T>(S, ld, k, t0 + I, t0 + J);
}

// one output tile (gI, gJ), gI >= gJ
template <typename T>
static __global__ void __launch_bounds__(256) syrk_cc_tile_kernel(T* __restrict__ S, int ld, int k, int gI, int gJ,
                                                                  const int* __restrict__ active) {
  if (active && !*active) return;
  syrk_cc_tile<T>(S, ld, k, gI, gJ);
}

template <typename T>
__device__ inline void syrk_cc_tile(T* __restrict__ S, int ld, int k, int gI, int gJ) {
  constexpr int KC = 16;
  __shared__ T As[KC][NB + 4];
  __shared__ T Bs[KC][NB + 4];
  const int I = gI, J = gJ;
  const int rA = gI * NB, rB = gJ * NB, kc = k * NB;
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
// 512 threads: warp w owns rows 8w..8w+7 of a 128-row tile, lane l owns
// columns 4l..4l+3; partial dot products stay in registers across tiles and
// are reduced once.
// Flags are read with GPU-scope acquire loads and written with release
// stores: the acquire that sees a tile's flag orders the waiting CTA's later
// reads of that tile (after its barrier) behind the tile's writes.
__device__ inline int load_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
static __device__ inline bool wait_flag(const int* flag, int epoch, int* status, long long limit) {
  long long it = 0;
  while (load_acquire(flag) != epoch) {
    if (++it > limit) {
      atomicOr(status, ST_SPIN_TIMEOUT);
      return false;
    }
    if (it > 4096) __nanosleep(100);
  }
  return true;
}

// Publish a solved tile: the barrier orders every thread's writes of the
// tile before thread 0's release store of the flag, which by cumulativity
// orders them before the flag for every observer (one release per CTA).
__device__ inline void publish_tile(int* flag, int epoch, int tid) {
  __syncthreads();
  if (tid == 0) asm volatile("st.release.gpu.global.b32 [%0], %1;\n" ::"l"(flag), "r"(epoch) : "memory");
}

static __global__ void set_int_kernel(int* p, int v) { *p = v; }

template <typename T>
__device__ inline void load4(const T* p, double* v) {
  if (sizeof(T) == 4) {
    const float4 f = *reinterpret_cast<const float4*>(p);
    v[0] = f.x; v[1] = f.y; v[2] = f.z; v[3] = f.w;
  } else {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
}

__device__ inline void load4_cg(const double* p, double* v) {
  const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldcg(reinterpret_cast<const double2*>(p + 2));
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

constexpr int SV = 512;
template <typename T>
constexpr size_t trsv_smem() {
  return sizeof(T) * NB * NB;
}

// Four consecutive entries of an L row in the storage type (kept raw in
// registers, widened to FP64 at the product).
template <typename T>
struct Row4;
template <>
struct Row4<float> {
  float4 v;
  __device__ __forceinline__ void load(const float* p) { v = *reinterpret_cast<const float4*>(p); }
  __device__ __forceinline__ double dot(const double* y) const {
    return (double)v.x * y[0] + (double)v.y * y[1] + (double)v.z * y[2] + (double)v.w * y[3];
  }
  __device__ __forceinline__ double at(int q) const {
    return q == 0 ? (double)v.x : q == 1 ? (double)v.y : q == 2 ? (double)v.z : (double)v.w;
  }
};
template <>
struct Row4<double> {
  double2 a, b;
  __device__ __forceinline__ void load(const double* p) {
    a = reinterpret_cast<const double2*>(p)[0];
    b = reinterpret_cast<const double2*>(p)[1];
  }
  __device__ __forceinline__ double dot(const double* y) const { return a.x * y[0] + a.y * y[1] + b.x * y[2] + b.y * y[3]; }
  __device__ __forceinline__ double at(int q) const { return q == 0 ? a.x : q == 1 ? a.y : q == 2 ? b.x : b.y; }
};

// Sums over the 32 lanes of eight per-lane values v[0..7] by recursive
// halving: at offsets 16, 8 and 4 each lane keeps half of its values and adds
// its partner's copy of them, then two butterfly steps finish.  Lane l ends
// with the full sum of v[4 b4 + 2 b3 + b2] (b4, b3, b2 = bits 4, 3, 2 of l;
// `reduce8_row` gives that index).  9 exchanges, 5 dependent levels; the
// order of the additions is fixed by the lane numbers.
__device__ __forceinline__ int reduce8_row(int lane) {
  return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
}
__device__ __forceinline__ double reduce8(const double (&v)[8], int lane) {
  const bool h4 = lane & 16, h3 = lane & 8, h2 = lane & 4;
  double a[4], b[2];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const double send = h4 ? v[q] : v[4 + q];
    a[q] = (h4 ? v[4 + q] : v[q]) + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const double send = h3 ? a[q] : a[2 + q];
    b[q] = (h3 ? a[2 + q] : a[q]) + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  double c = (h2 ? b[1] : b[0]) + __shfl_xor_sync(0xffffffffu, h2 ? b[0] : b[1], 4);
  c += __shfl_xor_sync(0xffffffffu, c, 2);
  c += __shfl_xor_sync(0xffffffffu, c, 1);
  return c;
}

// The tiles a solve CTA reads before its own are published in ticket order,
// so one wait is followed by a scan of the next flags: every tile found
// published joins the confirmed range, which the CTA then streams without
// further waits or barriers.  Thread 0 waits (bounded) on flag J and scans
// forward (step +1, up to `end` exclusive) or backward (step -1); the result
// is the first tile not confirmed, or `fail` after a timed-out wait.  The
// acquire loads of thread 0 followed by the caller's barrier order every
// thread's later reads of the confirmed tiles.
__device__ inline int confirm_tiles(const int* flags, int J, int end, int step, int epoch, int* status,
                                    long long limit, int fail) {
  if (!wait_flag(flags + J, epoch, status, limit)) return fail;
  int r = J + step;
  while (r != end && load_acquire(flags + r) == epoch) r += step;
  return r;
}

// The hop matrices of the solves, formed once per factorisation.  For the
// d-th neighbour (d = 1 .. kHopDepth):
//   M_d,I = Linv_I L_I,I-d                 (forward, I >= d)
//   Q_d,I = (L_I+d,I Linv_I)'              (backward, I + d < ntiles)
// at hop + ((dir kHopDepth + d - 1) ntiles + I) NB^2, dir 0 forward / 1
// backward.  With them y_I = c_I - sum_d M_d,I y_I-d, where c_I = Linv_I (b_I
// - sum_{J < I - kHopDepth} L_IJ y_J) needs only tiles published kHopDepth
// hops earlier, and likewise x_I = c'_I - sum_d Q_d,I x_I+d: after the wait
// for its neighbour a solve CTA applies one register-resident 128 x 128
// matrix.  Grid (ntiles - 1, 2 kHopDepth); products in T (FP32 for the mixed
// factor, FP64 for the FP64 one), 8 x 8 outputs per thread.  A tile L outside
// the envelope is zero, and so is its hop matrix.
constexpr int kHopDepth = 2;
template <typename T>
static __global__ void __launch_bounds__(256) hop_mat_kernel(const T* __restrict__ S, int ld, int ntiles,
                                                            const T* __restrict__ Linv, T* __restrict__ hop,
                                                            const int* __restrict__ active) {
  constexpr int KC = 16;
  __shared__ T As[KC][NB + 4];  // As[k][r] = A[r][k0 + k]
  __shared__ T Bs[KC][NB + 4];  // Bs[k][c] = B[k0 + k][c]
  if (active && !*active) return;
  const bool fwd = blockIdx.y < kHopDepth;
  const int d = (int)(blockIdx.y % kHopDepth) + 1;
  // forward: I = d + x, tile (I, I - d); backward: I = x, tile (I + d, I)
  const int I = fwd ? d + (int)blockIdx.x : (int)blockIdx.x;
  if ((fwd && I >= ntiles) || (!fwd && I + d >= ntiles)) return;
  const T* Lt = fwd ? S + (size_t)I * NB * ld + (size_t)(I - d) * NB : S + (size_t)(I + d) * NB * ld + (size_t)I * NB;
  const T* A = fwd ? Linv + (size_t)I * NB * NB : Lt;
  const size_t lda = fwd ? NB : (size_t)ld;
  const T* B = fwd ? Lt : Linv + (size_t)I * NB * NB;
  const size_t ldb = fwd ? (size_t)ld : NB;
  T* out = hop + ((size_t)blockIdx.y * ntiles + I) * NB * NB;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = (T)0;
  for (int k0 = 0; k0 < NB; k0 += KC) {
    for (int e = tid; e < NB * KC; e += 256) {
      const int r = e / KC, kk = e - r * KC;
      As[kk][r] = A[(size_t)r * lda + k0 + kk];
      const int kb = e / NB, c = e - kb * NB;
      Bs[kb][c] = B[(size_t)(k0 + kb) * ldb + c];
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < KC; kk++) {
      T a[8], bb[8];
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 8; j++) bb[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] += a[i] * bb[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int r = ty + 16 * i, c = tx + 16 * j;
      if (fwd)
        out[(size_t)r * NB + c] = acc[i][j];
      else
        out[(size_t)c * NB + r] = acc[i][j];
    }
}

// Forward solve L y = b by 128-row tiles.  CTA I (ticket order): streams the
// tiles J < I - kHopDepth of its row as they are published, forms c_I =
// Linv_I (b_I - partial) while its neighbours are still being solved, then
// subtracts M_d,I y_I-d for d = kHopDepth .. 1, each as soon as that tile is
// published.  Thread (warp w, lane l) holds rows 8 w .. 8 w + 7, columns
// 4 l .. 4 l + 3 of every 128 x 128 block it applies.
template <typename T>
static __global__ void __launch_bounds__(SV) trsv_fwd_kernel(const T* __restrict__ L, int ld, int ntiles,
                                                             const T* __restrict__ Linv,
                                                             const T* __restrict__ hop,
                                                             const double* __restrict__ b, double* __restrict__ y,
                                                             int* __restrict__ ticket, int* __restrict__ flags,
                                                             int epoch, int* __restrict__ status,
                                                             long long spin_limit,
                                                             const int* __restrict__ env,
                                                             const int* __restrict__ active) {
  extern __shared__ float4 sLi4[];
  T* sLi = reinterpret_cast<T*>(sLi4);  // Linv_I, NB x NB
  __shared__ double acc[NB];
  __shared__ int I_s, rdy_s[2];
  if (active && !*active) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) I_s = atomicAdd(ticket, 1);
  __syncthreads();
  const int I = I_s;
  {
    const float4* src = reinterpret_cast<const float4*>(Linv + (size_t)I * NB * NB);
    float4* dst = sLi4;
    for (int i = tid; i < (int)(NB * NB * sizeof(T) / 16); i += SV) dst[i] = src[i];
  }
  double part[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const T* Lrow = L + (size_t)(I * NB + warp * 8) * ld + 4 * lane;
  // the right-hand side of the row this lane finishes, loaded now
  const int rsel = warp * 8 + reduce8_row(lane);
  const double b_own = b[(size_t)I * NB + rsel];
  // with an envelope, the tiles of row I before its first nonzero are zero
  const int J0 = env ? env[I] : 0;
  const int Jend = I - kHopDepth;  // tiles [J0, Jend) are streamed, the last kHopDepth go through M_d,I
  constexpr bool kPre = sizeof(T) == 4;  // FP32: the next tile loads while this one is used
  Row4<T> cur[8], nxt[8];
  if (J0 < Jend) {
#pragma unroll
    for (int rr = 0; rr < 8; rr++) cur[rr].load(Lrow + (size_t)rr * ld + (size_t)J0 * NB);
  }
  int ready = J0, par = 0;  // tiles [J0, ready) are confirmed published
  auto catch_up = [&](int J) -> bool {  // uniform: every thread calls it with the same J
    if (tid == 0) rdy_s[par] = confirm_tiles(flags, J, I, 1, epoch, status, spin_limit, -1);
    __syncthreads();
    ready = rdy_s[par];
    par ^= 1;  // the other slot is written only after the next barrier
    return ready >= 0;
  };
  for (int J = J0; J < Jend; J++) {
    if (kPre && J + 1 < Jend) {
#pragma unroll
      for (int rr = 0; rr < 8; rr++) nxt[rr].load(Lrow + (size_t)rr * ld + (size_t)(J + 1) * NB);
    }
    if (J >= ready && !catch_up(J)) return;
    double yv[4];
    load4_cg(y + (size_t)J * NB + 4 * lane, yv);
#pragma unroll
    for (int rr = 0; rr < 8; rr++) part[rr] += cur[rr].dot(yv);
    if (kPre) {
#pragma unroll
      for (int rr = 0; rr < 8; rr++) cur[rr] = nxt[rr];
    } else if (J + 1 < Jend) {
#pragma unroll
      for (int rr = 0; rr < 8; rr++) cur[rr].load(Lrow + (size_t)rr * ld + (size_t)(J + 1) * NB);
    }
  }
  // c_I = Linv_I (b_I - partial)
  {
    const double sr = reduce8(part, lane);
    if ((lane & 3) == 0) acc[rsel] = b_own - sr;
  }
  __syncthreads();
  const T* Li = sLi + (size_t)(warp * 8) * NB + 4 * lane;
  double av[4] = {acc[4 * lane], acc[4 * lane + 1], acc[4 * lane + 2], acc[4 * lane + 3]};
  double q8[8];
#pragma unroll
  for (int rr = 0; rr < 8; rr++) {
    double lv[4];
    load4(Li + (size_t)rr * NB, lv);
    q8[rr] = lv[0] * av[0] + lv[1] * av[1] + lv[2] * av[2] + lv[3] * av[3];
  }
  double yr = reduce8(q8, lane);
  // y_I = c_I - sum_d M_d,I y_I-d, nearest tile last
#pragma unroll
  for (int d = kHopDepth; d >= 1; d--) {
    const int J = I - d;
    if (J < 0 || J < J0) continue;  // outside the matrix or the envelope (uniform)
    Row4<T> mrow[8];
    const T* Mr = hop + ((size_t)(d - 1) * ntiles + I) * NB * NB + (size_t)(warp * 8) * NB + 4 * lane;
#pragma unroll
    for (int rr = 0; rr < 8; rr++) mrow[rr].load(Mr + (size_t)rr * NB);
    if (J >= ready && !catch_up(J)) return;
    double yv[4];
    load4_cg(y + (size_t)J * NB + 4 * lane, yv);
#pragma unroll
    for (int rr = 0; rr < 8; rr++) q8[rr] = mrow[rr].dot(yv);
    yr -= reduce8(q8, lane);
  }
  if ((lane & 3) == 0) y[(size_t)I * NB + rsel] = yr;
  publish_tile(flags + I, epoch, tid);
}

// Backward solve L' x = y.  CTA I (reverse ticket order): streams the tiles
// J > I + kHopDepth of column I (rows of L_J,I) as they are published, forms
// c'_I = Linv_I' (y_I - partial), then subtracts Q_d,I x_I+d for
// d = kHopDepth .. 1 (Q_d,I row-major: row c is column c of L_I+d,I Linv_I,
// so these steps have the forward kernel's row layout).
template <typename T>
static __global__ void __launch_bounds__(SV) trsv_bwd_kernel(const T* __restrict__ L, int ld, int ntiles,
                                                             const T* __restrict__ Linv,
                                                             const T* __restrict__ hop,
                                                             const double* __restrict__ yv, double* __restrict__ x,
                                                             int* __restrict__ ticket, int* __restrict__ flags,
                                                             int epoch, int* __restrict__ status,
                                                             long long spin_limit,
                                                             const int* __restrict__ env,
                                                             const int* __restrict__ active) {
  extern __shared__ float4 sLi4[];
  T* sLi = reinterpret_cast<T*>(sLi4);  // Linv_I, NB x NB
  __shared__ double red[SV / 32][NB];
  __shared__ double acc[NB];
  __shared__ int I_s, rdy_s[2];
  if (active && !*active) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) I_s = ntiles - 1 - atomicAdd(ticket, 1);
  __syncthreads();
  const int I = I_s;
  {
    const float4* src = reinterpret_cast<const float4*>(Linv + (size_t)I * NB * NB);
    float4* dst = sLi4;
    for (int i = tid; i < (int)(NB * NB * sizeof(T) / 16); i += SV) dst[i] = src[i];
  }
  double part[4] = {0, 0, 0, 0};
  const double y_own = tid < NB ? yv[(size_t)I * NB + tid] : 0.0;  // loaded off the chain
  // with an envelope, the tiles of column I past its last nonzero are zero
  const int J1 = env ? env[ntiles + I] : ntiles - 1;
  const int Jend = I + kHopDepth;  // tiles (Jend, J1] are streamed, the nearest kHopDepth go through Q_d,I
  const T* Lcol = L + (size_t)(warp * 8) * ld + (size_t)I * NB + 4 * lane;  // + J NB ld: tile (J, I)
  constexpr bool kPre = sizeof(T) == 4;
  Row4<T> cur[8], nxt[8];
  if (J1 > Jend) {
#pragma unroll
    for (int rr = 0; rr < 8; rr++) cur[rr].load(Lcol + (size_t)(J1 * NB + rr) * ld);
  }
  int lo = J1 + 1, par = 0;  // tiles [lo, J1] are confirmed published
  auto catch_up = [&](int J) -> bool {  // uniform
    if (tid == 0) rdy_s[par] = confirm_tiles(flags, J, I, -1, epoch, status, spin_limit, -1) + 1;
    __syncthreads();
    lo = rdy_s[par];
    par ^= 1;
    return lo > 0;
  };
  for (int J = J1; J > Jend; J--) {
    if (kPre && J - 1 > Jend) {
#pragma unroll
      for (int rr = 0; rr < 8; rr++) nxt[rr].load(Lcol + (size_t)((J - 1) * NB + rr) * ld);
    }
    if (J < lo && !catch_up(J)) return;
#pragma unroll
    for (int rr = 0; rr < 8; rr++) {
      const double xr = __ldcg(x + (size_t)J * NB + warp * 8 + rr);
#pragma unroll
      for (int q = 0; q < 4; q++) part[q] += cur[rr].at(q) * xr;
    }
    if (kPre) {
#pragma unroll
      for (int rr = 0; rr < 8; rr++) cur[rr] = nxt[rr];
    } else if (J - 1 > Jend) {
#pragma unroll
      for (int rr = 0; rr < 8; rr++) cur[rr].load(Lcol + (size_t)((J - 1) * NB + rr) * ld);
    }
  }
#pragma unroll
  for (int q = 0; q < 4; q++) red[warp][4 * lane + q] = part[q];
  __syncthreads();
  if (tid < NB) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < SV / 32; w++) s += red[w][tid];
    acc[tid] = y_own - s;
  }
  __syncthreads();
  // c'_I = Linv_I' acc : c'[c] = sum_r Linv[r][c] acc[r]
  const T* Li = sLi + (size_t)(warp * 8) * NB + 4 * lane;
  double p2[4] = {0, 0, 0, 0};
#pragma unroll
  for (int rr = 0; rr < 8; rr++) {
    const double ar = acc[warp * 8 + rr];
    double lv[4];
    load4(Li + (size_t)rr * NB, lv);
    p2[0] += lv[0] * ar;
    p2[1] += lv[1] * ar;
    p2[2] += lv[2] * ar;
    p2[3] += lv[3] * ar;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; q++) red[warp][4 * lane + q] = p2[q];
  __syncthreads();
  if (tid < NB) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < SV / 32; w++) s += red[w][tid];
    acc[tid] = s;  // c'_I
  }
  __syncthreads();
  const int rsel = warp * 8 + reduce8_row(lane);
  double xr = acc[rsel];
  // x_I = c'_I - sum_d Q_d,I x_I+d, nearest tile last
#pragma unroll
  for (int d = kHopDepth; d >= 1; d--) {
    const int J = I + d;
    if (J >= ntiles || J > J1) continue;  // outside the matrix or the envelope (uniform)
    Row4<T> qrow[8];
    const T* Qr = hop + ((size_t)(kHopDepth + d - 1) * ntiles + I) * NB * NB + (size_t)(warp * 8) * NB + 4 * lane;
#pragma unroll
    for (int rr = 0; rr < 8; rr++) qrow[rr].load(Qr + (size_t)rr * NB);
    if (J < lo && !catch_up(J)) return;
    double xv[4];
    load4_cg(x + (size_t)J * NB + 4 * lane, xv);
    double q8[8];
#pragma unroll
    for (int rr = 0; rr < 8; rr++) q8[rr] = qrow[rr].dot(xv);
    xr -= reduce8(q8, lane);
  }
  if ((lane & 3) == 0) x[(size_t)I * NB + rsel] = xr;
  publish_tile(flags + I, epoch, tid);
}

// ---------------------------------------------------------------------------
// Refinement residual r = b - S0 x from the lower storage of S0.  Grid
// (row tile I, chunk); a chunk covers a range of column tiles J.  For J < I
// the tile S0_IJ is read row-wise (y_I += S0_IJ x_J), for J > I the tile
// S0_JI is read row-wise and applied transposed (y_I += S0_JI' x_J); the
// diagonal tile uses both halves.  Partials per chunk are summed in a fixed
// order by resid_finalize_kernel.
template <typename T, int NCH>
static __global__ void __launch_bounds__(SV) symv_partial_kernel(const T* __restrict__ S0, int ld, int ntiles,
                                                                 const double* __restrict__ x,
                                                                 double* __restrict__ part,
                                                                 const int* __restrict__ active) {
  __shared__ double red[SV / 32][NB];
  if (active && !*active) return;
  const int I = blockIdx.x, ch = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = (ntiles + NCH - 1) / NCH;
  const int J0 = ch * per, J1 = min(ntiles, J0 + per);
  double rp[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // rows 8 warp + rr
  double cp[4] = {0, 0, 0, 0};              // columns 4 lane + q
  for (int J = J0; J < J1; J++) {
    if (J <= I) {
      const T* Ls = S0 + (size_t)(I * NB + warp * 8) * ld + (size_t)J * NB + 4 * lane;
      double xv[4];
      load4(x + (size_t)J * NB + 4 * lane, xv);
#pragma unroll
      for (int rr = 0; rr < 8; rr++) {
        double lv[4];
        load4(Ls + (size_t)rr * ld, lv);
        if (J == I) {  // lower half of the diagonal tile: c <= r
          const int r = warp * 8 + rr;
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (4 * lane + q > r) lv[q] = 0.0;
        }
        rp[rr] += lv[0] * xv[0] + lv[1] * xv[1] + lv[2] * xv[2] + lv[3] * xv[3];
      }
    }
    if (J >= I) {
      const T* Ls = S0 + (size_t)(J * NB + warp * 8) * ld + (size_t)I * NB + 4 * lane;
#pragma unroll
      for (int rr = 0; rr < 8; rr++) {
        const int r = warp * 8 + rr;  // row of tile J
        const double xr = x[(size_t)J * NB + r];
        double lv[4];
        load4(Ls + (size_t)rr * ld, lv);
        if (J == I) {  // strictly-lower entries (r > c) applied transposed
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (r <= 4 * lane + q) lv[q] = 0.0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) cp[q] += lv[q] * xr;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 4; q++) red[warp][4 * lane + q] = cp[q];
  __syncthreads();
  double rowsum[8];
#pragma unroll
  for (int rr = 0; rr < 8; rr++) rowsum[rr] = warp_sum(rp[rr]);
  if (lane == 0) {
#pragma unroll
    for (int rr = 0; rr < 8; rr++) {
      const int r = warp * 8 + rr;
      double c = 0.0;
#pragma unroll
      for (int w = 0; w < SV / 32; w++) c += red[w][r];
      part[(size_t)ch * ntiles * NB + (size_t)I * NB + r] = rowsum[rr] + c;
    }
  }
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
