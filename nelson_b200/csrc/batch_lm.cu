// batch_lm.cu -- many independent small BA problems in one persistent launch.
//
// LevenbergMarquardt<SolverCholeskySchur>::solve
// (nelson/LevenbergMarquardt.hpp:36-146, nelson/SolverCholeskySchur.hpp:91-157)
// for n problems of uneven sizes at once: one kernel launch whose CTAs take
// problems from a device work queue (an atomic counter over the problems in
// descending order of estimated work) and run each problem's whole LM solve,
// sub-iteration by sub-iteration, with the CTA's threads:
//   update(true)     cost, then V / bV / W per variable point (one thread per
//                    point over its edges) and U / bU per camera (one warp per
//                    camera over its edges, butterfly reduction);
//   computeIncrement damped V^-1, xV0 = -V^-1 bV and Y = W V^-1 per point;
//                    bS = -bU - W xV0 per camera; S = U - sum Y W' block by
//                    block over (Y, W) edge pairs of a common point (one warp
//                    per block, points ascending), damping on the diagonal;
//                    blocked Cholesky of S (32-column panels staged in shared
//                    memory, 4 x 4 register tiles for the trailing update);
//                    forward / backward solves by 32-row blocks; back-
//                    substitution per point;
//   the LM decisions (gain ratio, accept / reject, damping, termination) on
//                    one thread, exactly as the reference orders them.
// Everything is FP64.  No CTA ever waits for another, so nothing can hang;
// every loop is bounded by the problem sizes and the LM iteration limits.
// Every sum has a fixed order that does not depend on the CTA size or on which
// CTA takes the problem (per-thread loops, warp butterflies, 32-element chunk
// sums added in order), so a problem's result does not depend on the launch
// shape or on the other problems of the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <vector>

#include "ba_kernels.cuh"
#include "problem_view.h"
#include "schur_core.cuh"

namespace nl {
namespace {

constexpr int kPW = 32;         // Cholesky / solve panel width
constexpr int kPLd = kPW + 1;   // shared panel row stride (doubles)
constexpr int kMaxN = 768;      // largest reduced camera system of the persistent path

struct BProb {
  int ncv, nc_all, npv, np_all, ne, n, nS, pad;
  double f, cx, cy;
  const int* e_cam;     // E-order edges: camera slot (variable: user index; fixed: ncv + index)
  const int* e_pt;      // point slot (variable: index; fixed: npv + index)
  const double* e_obs;  // 2 per edge
  const double* e_w;
  const int* cam_ptr;   // ncv + 1: E-order edges of internal camera c
  const int* cam_slot;  // internal camera -> slot
  const int* slot2int;  // camera slot -> internal camera, -1 for a fixed camera
  const int* pt_ptr;    // npv + 1: P-order edges of point p
  const int* p2e;       // P-order -> E-order
  const int* s_i;       // S blocks (i <= j, internal cameras)
  const int* s_j;
  const int* s_ptr;     // nS + 1: pairs of block b
  const int* pa;        // pair: E-order edge of camera i
  const int* pb;        // pair: E-order edge of camera j, same point
  double* cam;          // nc_all x 16 camera state
  double* pt;           // np_all x 3
  double* cam_bck;
  double* pt_bck;
  double* W;            // ne x BC*3 (edges with a variable camera and a variable point)
  double* Y;            // ne x BC*3
  double* U;            // ncv x BC*BC (internal order)
  double* bU;           // ncv x BC
  double* V;            // npv x 9
  double* Vinv;         // npv x 9
  double* bV;           // npv x 3
  double* xV0;          // npv x 3
  double* S;            // n x n (lower triangle used)
  double* bS;           // n
  double* inc;          // n + 3 npv: internal camera order, then points
  double* part;         // chunk partials
};

struct BSettings {
  int maxNumIt, maxNumSubIt, minNumIt, pad;
  double epsBVector, epsIncSquare, epsChi2, tau, penaltyV, initV, maxScale, minScale;
};

struct BReport {
  int reason, iterations, subiterations, pad;
  double chi2, mu;
  unsigned long long t_start, t_end;  // %globaltimer (ns)
};

struct LmS {
  double mu, curV, oldChi2, chi2, chi2_new, rho, incSq, den, maxAbsB;
  int iter, subiter, nsub, done, reason, ok, apply, acc;
};

__device__ inline unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ inline double warp_all_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// sum_{i < cnt} f(i) in an order fixed by cnt alone: 32-element chunks summed
// by a warp butterfly, chunk sums added by warp 0 in a fixed pattern.  Every
// thread gets the result.
template <class F>
__device__ double cta_sum(int cnt, F f, double* part, double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int nch = (cnt + 31) / 32;
  for (int c = warp; c < nch; c += nw) {
    const int i = c * 32 + lane;
    const double v = warp_all_sum(i < cnt ? f(i) : 0.0);
    if (lane == 0) part[c] = v;
  }
  __syncthreads();
  if (warp == 0) {
    double v = 0.0;
    for (int c = lane; c < nch; c += 32) v += part[c];
    v = warp_all_sum(v);
    if (lane == 0) sh[0] = v;
  }
  __syncthreads();
  const double r = sh[0];
  __syncthreads();
  return r;
}

// max_{i < cnt} f(i) (exact in any order).
template <class F>
__device__ double cta_max(int cnt, F f, double* sh) {
  double m = 0.0;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) m = fmax(m, f(i));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) r = fmax(r, sh[w]);
    sh[32] = r;
  }
  __syncthreads();
  const double r = sh[32];
  __syncthreads();
  return r;
}

// Sums the 36 per-lane values v over the warp by recursive halving (a
// reduce-scatter): at offsets 16, 8, 4, 2, 1 each lane keeps half of its
// values (odd counts padded with a zero) and adds its partner's copy of them.
// 37 exchanges instead of 36 butterflies of 5.  Lane l ends with two sums,
// out[i] of entry idx[i] (-1 for a padding slot); every entry lands on
// exactly one lane, and the order of the additions depends on the lane
// numbers alone.
__device__ inline void reduce_scatter36(const double (&v)[36], int lane, double (&out)[2], int (&idx)[2]) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2, b0 = lane & 1;
  double a[18];
#pragma unroll
  for (int i = 0; i < 18; i++)
    a[i] = (b4 ? v[18 + i] : v[i]) + __shfl_xor_sync(0xffffffffu, b4 ? v[i] : v[18 + i], 16);
  double c[10];
#pragma unroll
  for (int i = 0; i < 9; i++)
    c[i] = (b3 ? a[9 + i] : a[i]) + __shfl_xor_sync(0xffffffffu, b3 ? a[i] : a[9 + i], 8);
  c[9] = 0.0;
  double d[6];
#pragma unroll
  for (int i = 0; i < 5; i++)
    d[i] = (b2 ? c[5 + i] : c[i]) + __shfl_xor_sync(0xffffffffu, b2 ? c[i] : c[5 + i], 4);
  d[5] = 0.0;
  double f[4];
#pragma unroll
  for (int i = 0; i < 3; i++)
    f[i] = (b1 ? d[3 + i] : d[i]) + __shfl_xor_sync(0xffffffffu, b1 ? d[i] : d[3 + i], 2);
  f[3] = 0.0;
#pragma unroll
  for (int i = 0; i < 2; i++) {
    out[i] = (b0 ? f[2 + i] : f[i]) + __shfl_xor_sync(0xffffffffu, b0 ? f[i] : f[2 + i], 1);
    const int l1 = 2 * b0 + i, l2 = 3 * b1 + l1, l3 = 5 * b2 + l2;
    idx[i] = (l1 < 3 && l2 < 5 && l3 < 9) ? 18 * b4 + 9 * b3 + l3 : -1;
  }
}

template <int BC>
__device__ double cost(const BProb& P, double* sh) {
  return cta_sum(
      P.ne,
      [&](int e) {
        double r0, r1;
        ba_project<double, BC, false, false>(P.cam + (size_t)P.e_cam[e] * 16, P.pt + (size_t)P.e_pt[e] * 3,
                                             P.e_obs[2 * e], P.e_obs[2 * e + 1], P.f, P.cx, P.cy, r0, r1, nullptr,
                                             nullptr);
        return P.e_w[e] * (r0 * r0 + r1 * r1);
      },
      P.part, sh);
}

// update(true) without the cost: V, bV, W (points) and U, bU (cameras).
template <int BC>
__device__ void jacobian_pass(const BProb& P) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  for (int p = tid; p < P.npv; p += nt) {
    double v[6] = {0, 0, 0, 0, 0, 0}, b[3] = {0, 0, 0};
    for (int t = P.pt_ptr[p]; t < P.pt_ptr[p + 1]; t++) {
      const int e = P.p2e[t];
      const int cs = P.e_cam[e];
      double r0, r1, Jc[2 * BC], Jp[6];
      ba_project<double, BC, true, true>(P.cam + (size_t)cs * 16, P.pt + (size_t)p * 3, P.e_obs[2 * e],
                                         P.e_obs[2 * e + 1], P.f, P.cx, P.cy, r0, r1, Jc, Jp);
      const double w = P.e_w[e];
      int q = 0;
#pragma unroll
      for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = i; j < 3; j++) v[q++] += w * (Jp[i] * Jp[j] + Jp[3 + i] * Jp[3 + j]);
        b[i] += w * (Jp[i] * r0 + Jp[3 + i] * r1);
      }
      if (cs < P.ncv) {
        double* We = P.W + (size_t)e * (BC * 3);
#pragma unroll
        for (int i = 0; i < BC; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) We[i * 3 + j] = w * (Jc[i] * Jp[j] + Jc[BC + i] * Jp[3 + j]);
      }
    }
    double* Vp = P.V + (size_t)p * 9;
    Vp[0] = v[0]; Vp[1] = v[1]; Vp[2] = v[2];
    Vp[3] = v[1]; Vp[4] = v[3]; Vp[5] = v[4];
    Vp[6] = v[2]; Vp[7] = v[4]; Vp[8] = v[5];
    P.bV[3 * (size_t)p] = b[0];
    P.bV[3 * (size_t)p + 1] = b[1];
    P.bV[3 * (size_t)p + 2] = b[2];
  }
  constexpr int NUU = BC * (BC + 1) / 2;
  for (int c = warp; c < P.ncv; c += nw) {
    const double* cs = P.cam + (size_t)P.cam_slot[c] * 16;
    double u[NUU], b[BC];
#pragma unroll
    for (int i = 0; i < NUU; i++) u[i] = 0.0;
#pragma unroll
    for (int i = 0; i < BC; i++) b[i] = 0.0;
    for (int e = P.cam_ptr[c] + lane; e < P.cam_ptr[c + 1]; e += 32) {
      double r0, r1, Jc[2 * BC];
      ba_project<double, BC, true, false>(cs, P.pt + (size_t)P.e_pt[e] * 3, P.e_obs[2 * e], P.e_obs[2 * e + 1], P.f,
                                          P.cx, P.cy, r0, r1, Jc, nullptr);
      const double w = P.e_w[e];
      int q = 0;
#pragma unroll
      for (int i = 0; i < BC; i++) {
#pragma unroll
        for (int j = i; j < BC; j++) u[q++] += w * (Jc[i] * Jc[j] + Jc[BC + i] * Jc[BC + j]);
        b[i] += w * (Jc[i] * r0 + Jc[BC + i] * r1);
      }
    }
#pragma unroll
    for (int i = 0; i < NUU; i++) u[i] = warp_all_sum(u[i]);
#pragma unroll
    for (int i = 0; i < BC; i++) b[i] = warp_all_sum(b[i]);
    if (lane == 0) {
      double* Uc = P.U + (size_t)c * BC * BC;
      int q = 0;
#pragma unroll
      for (int i = 0; i < BC; i++)
#pragma unroll
        for (int j = i; j < BC; j++) {
          Uc[i * BC + j] = u[q];
          Uc[j * BC + i] = u[q];
          q++;
        }
#pragma unroll
      for (int i = 0; i < BC; i++) P.bU[(size_t)c * BC + i] = b[i];
    }
  }
}

// (V_p + mu I)^-1 by Cholesky; false if not positive definite.
__device__ inline bool spd3_inverse(const double* A, double mu, double* X) {
  const double a00 = A[0] + mu, a10 = A[3], a11 = A[4] + mu, a20 = A[6], a21 = A[7], a22 = A[8] + mu;
  if (!(a00 > 0.0)) return false;
  const double l00 = sqrt(a00);
  const double l10 = a10 / l00, l20 = a20 / l00;
  const double d1 = a11 - l10 * l10;
  if (!(d1 > 0.0)) return false;
  const double l11 = sqrt(d1);
  const double l21 = (a21 - l20 * l10) / l11;
  const double d2 = a22 - l20 * l20 - l21 * l21;
  if (!(d2 > 0.0) || !isfinite(d2)) return false;
  const double l22 = sqrt(d2);
  // inv(L)
  const double i00 = 1.0 / l00, i11 = 1.0 / l11, i22 = 1.0 / l22;
  const double i10 = -l10 * i00 * i11;
  const double i21 = -l21 * i11 * i22;
  const double i20 = -(l20 * i00 + l21 * i10) * i22;
  // X = inv(L)' inv(L)
  X[0] = i00 * i00 + i10 * i10 + i20 * i20;
  X[1] = i10 * i11 + i20 * i21;
  X[2] = i20 * i22;
  X[4] = i11 * i11 + i21 * i21;
  X[5] = i21 * i22;
  X[8] = i22 * i22;
  X[3] = X[1];
  X[6] = X[2];
  X[7] = X[5];
  return true;
}

// computeIncrement(H, b, 0, mu): inc = [xU; xV].  Returns false when a damped
// point block or S is not positive definite (the increment is then zero).
template <int BC>
__device__ bool compute_increment(const BProb& P, double mu, double* smem, int* flag) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  const int n = P.n;
  if (tid == 0) *flag = 0;
  __syncthreads();
  // V^-1, xV0, Y per point
  for (int p = tid; p < P.npv; p += nt) {
    double* Vi = P.Vinv + (size_t)p * 9;
    if (!spd3_inverse(P.V + (size_t)p * 9, mu, Vi)) {
      *flag = 1;
      for (int i = 0; i < 9; i++) Vi[i] = 0.0;
    }
    const double* b = P.bV + (size_t)p * 3;
#pragma unroll
    for (int i = 0; i < 3; i++) P.xV0[3 * (size_t)p + i] = -(Vi[i * 3] * b[0] + Vi[i * 3 + 1] * b[1] + Vi[i * 3 + 2] * b[2]);
    for (int t = P.pt_ptr[p]; t < P.pt_ptr[p + 1]; t++) {
      const int e = P.p2e[t];
      if (P.e_cam[e] >= P.ncv) continue;
      const double* We = P.W + (size_t)e * (BC * 3);
      double* Ye = P.Y + (size_t)e * (BC * 3);
#pragma unroll
      for (int i = 0; i < BC; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
          Ye[i * 3 + j] = We[i * 3] * Vi[j] + We[i * 3 + 1] * Vi[3 + j] + We[i * 3 + 2] * Vi[6 + j];
    }
  }
  // the lower triangle of S starts from zero
  for (size_t i = tid; i < (size_t)n * n; i += nt) P.S[i] = 0.0;
  __syncthreads();
  // bS = -bU - W xV0 per camera
  for (int c = warp; c < P.ncv; c += nw) {
    double s[BC];
#pragma unroll
    for (int i = 0; i < BC; i++) s[i] = 0.0;
    for (int e = P.cam_ptr[c] + lane; e < P.cam_ptr[c + 1]; e += 32) {
      const int ps = P.e_pt[e];
      if (ps >= P.npv) continue;
      const double* We = P.W + (size_t)e * (BC * 3);
      const double* x = P.xV0 + (size_t)ps * 3;
#pragma unroll
      for (int i = 0; i < BC; i++) s[i] += We[i * 3] * x[0] + We[i * 3 + 1] * x[1] + We[i * 3 + 2] * x[2];
    }
#pragma unroll
    for (int i = 0; i < BC; i++) s[i] = warp_all_sum(s[i]);
    if (lane == 0)
#pragma unroll
      for (int i = 0; i < BC; i++) P.bS[(size_t)c * BC + i] = -P.bU[(size_t)c * BC + i] - s[i];
  }
  // S blocks: M = U_ij - sum_pairs Y_a W_b'
  constexpr int NE = BC * BC;
  for (int b = warp; b < P.nS; b += nw) {
    const int bi = P.s_i[b], bj = P.s_j[b];
    const int t0 = P.s_ptr[b], t1 = P.s_ptr[b + 1];
    if constexpr (BC == 6) {
      // lane l takes pairs l, l + 32, ... and accumulates the whole 6 x 6
      // product (32 pairs' loads in flight per warp); the lanes' sums are then
      // added by a butterfly, so the order depends on the pair count alone
      double acc[NE];
#pragma unroll
      for (int q = 0; q < NE; q++) acc[q] = 0.0;
      for (int t = t0 + lane; t < t1; t += 32) {
        const double2* Ya = reinterpret_cast<const double2*>(P.Y + (size_t)P.pa[t] * (BC * 3));
        const double2* Wb = reinterpret_cast<const double2*>(P.W + (size_t)P.pb[t] * (BC * 3));
        double y[BC * 3], w[BC * 3];
#pragma unroll
        for (int q = 0; q < BC * 3 / 2; q++) {
          const double2 a = Ya[q], c = Wb[q];
          y[2 * q] = a.x;
          y[2 * q + 1] = a.y;
          w[2 * q] = c.x;
          w[2 * q + 1] = c.y;
        }
#pragma unroll
        for (int r = 0; r < BC; r++)
#pragma unroll
          for (int c = 0; c < BC; c++)
            acc[r * BC + c] += y[r * 3] * w[c * 3] + y[r * 3 + 1] * w[c * 3 + 1] + y[r * 3 + 2] * w[c * 3 + 2];
      }
      double sum[2];
      int ent[2];
      reduce_scatter36(acc, lane, sum, ent);
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int q = ent[i];
        if (q >= 0) {
          const int r = q / BC, c = q % BC;
          double m = -sum[i];
          if (bi == bj) m += P.U[(size_t)bi * NE + q];
          // block (i, j) of the upper S at lower (j BC + c, i BC + r)
          const int row = bj * BC + c, col = bi * BC + r;
          if (col <= row) P.S[(size_t)row * n + col] = m;
        }
      }
    } else {
      // lane l owns entries l, l + 32, ...; four pairs' loads are issued
      // before their products
      constexpr int NPL = (NE + 31) / 32;
      double acc[NPL];
#pragma unroll
      for (int q = 0; q < NPL; q++) acc[q] = 0.0;
      int ra[NPL], ca[NPL];
#pragma unroll
      for (int q = 0; q < NPL; q++) {
        const int idx = min(lane + 32 * q, NE - 1);
        ra[q] = idx / BC;
        ca[q] = idx - (idx / BC) * BC;
      }
      for (int t = t0; t < t1; t += 4) {
        double yv[4][NPL][3], wv[4][NPL][3];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const bool in = t + u < t1;
          const double* Ya = P.Y + (size_t)(in ? P.pa[t + u] : P.pa[t0]) * (BC * 3);
          const double* Wb = P.W + (size_t)(in ? P.pb[t + u] : P.pb[t0]) * (BC * 3);
#pragma unroll
          for (int q = 0; q < NPL; q++)
#pragma unroll
            for (int k = 0; k < 3; k++) {
              yv[u][q][k] = in ? Ya[ra[q] * 3 + k] : 0.0;
              wv[u][q][k] = Wb[ca[q] * 3 + k];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
          for (int q = 0; q < NPL; q++)
            acc[q] += yv[u][q][0] * wv[u][q][0] + yv[u][q][1] * wv[u][q][1] + yv[u][q][2] * wv[u][q][2];
      }
#pragma unroll
      for (int q = 0; q < NPL; q++) {
        const int idx = lane + 32 * q;
        if (idx < NE) {
          double m = -acc[q];
          if (bi == bj) m += P.U[(size_t)bi * NE + idx];
          const int row = bj * BC + ca[q], col = bi * BC + ra[q];
          if (col <= row) P.S[(size_t)row * n + col] = m;
        }
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < n; i += nt) P.S[(size_t)i * n + i] += mu;
  __syncthreads();
  // blocked Cholesky: panel [k0, k0 + kb) of rows k0 .. n - 1 in shared memory
  for (int k0 = 0; k0 < n; k0 += kPW) {
    const int kb = min(kPW, n - k0), m = n - k0;
    for (int i = tid; i < m * kb; i += nt) {
      const int r = i / kb, c = i - (i / kb) * kb;
      smem[r * kPLd + c] = c <= r ? P.S[(size_t)(k0 + r) * n + k0 + c] : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < kb; j++) {
      double d = smem[j * kPLd + j];
      if (!(d > 0.0) || !isfinite(d)) {
        if (tid == 0) *flag = 1;
        d = 1.0;
      }
      const double ld = sqrt(d), il = 1.0 / ld;
      __syncthreads();  // every thread has read the pivot
      for (int r = j + 1 + tid; r < m; r += nt) smem[r * kPLd + j] *= il;
      if (tid == 0) smem[j * kPLd + j] = ld;
      __syncthreads();
      const int wc = kb - j - 1;
      if (wc > 0)
        for (int i = tid; i < (m - j - 1) * wc; i += nt) {
          const int r = j + 1 + i / wc, c = j + 1 + (i - (i / wc) * wc);
          if (c <= r) smem[r * kPLd + c] -= smem[r * kPLd + j] * smem[c * kPLd + j];
        }
      __syncthreads();
    }
    for (int i = tid; i < m * kb; i += nt) {
      const int r = i / kb, c = i - (i / kb) * kb;
      if (c <= r) P.S[(size_t)(k0 + r) * n + k0 + c] = smem[r * kPLd + c];
    }
    // trailing update of rows / columns k0 + kb .. n - 1, 4 x 4 register tiles
    const int tr = m - kb;
    if (tr > 0) {
      const int T4 = (tr + 3) / 4;
      const int ntile = T4 * (T4 + 1) / 2;
      for (int q = tid; q < ntile; q += nt) {
        int I = (int)((sqrtf(8.0f * q + 1.0f) - 1.0f) * 0.5f);
        while ((I + 1) * (I + 2) / 2 <= q) I++;
        while (I * (I + 1) / 2 > q) I--;
        const int J = q - I * (I + 1) / 2;
        double a[4][4];
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
          for (int v = 0; v < 4; v++) a[u][v] = 0.0;
        const int r0 = kb + 4 * I, c0 = kb + 4 * J;
        for (int jj = 0; jj < kb; jj++) {
          double x[4], y[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            x[u] = r0 + u < m ? smem[(r0 + u) * kPLd + jj] : 0.0;
            y[u] = c0 + u < m ? smem[(c0 + u) * kPLd + jj] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) a[u][v] += x[u] * y[v];
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const int r = r0 + u, c = c0 + v;
            if (r < m && c <= r) P.S[(size_t)(k0 + r) * n + k0 + c] -= a[u][v];
          }
      }
    }
    __syncthreads();
  }
  // forward solve L y = bS (y in inc[0, n))
  double* x = P.inc;
  for (int i = tid; i < n; i += nt) x[i] = P.bS[i];
  __syncthreads();
  for (int k0 = 0; k0 < n; k0 += kPW) {
    const int kb = min(kPW, n - k0);
    if (warp == 0) {
      // lane i holds row k0 + i of the diagonal block (independent loads first)
      double lrow[kPW];
#pragma unroll
      for (int j = 0; j < kPW; j++) lrow[j] = (lane < kb && j <= lane) ? P.S[(size_t)(k0 + lane) * n + k0 + j] : 0.0;
      double yi = lane < kb ? x[k0 + lane] : 0.0;
#pragma unroll
      for (int j = 0; j < kPW; j++) {
        if (j < kb) {
          const double djj = __shfl_sync(0xffffffffu, lrow[j], j);
          const double yj = __shfl_sync(0xffffffffu, yi, j) / djj;
          if (lane == j) yi = yj;
          if (lane > j && lane < kb) yi -= lrow[j] * yj;
        }
      }
      if (lane < kb) x[k0 + lane] = yi;
    }
    __syncthreads();
    for (int r = k0 + kb + tid; r < n; r += nt) {
      double s = x[r];
      const double* Lr = P.S + (size_t)r * n + k0;
      for (int j = 0; j < kb; j++) s -= Lr[j] * x[k0 + j];
      x[r] = s;
    }
    __syncthreads();
  }
  // backward solve L' x = y
  for (int k0 = ((n - 1) / kPW) * kPW; k0 >= 0 && n > 0; k0 -= kPW) {
    const int kb = min(kPW, n - k0);
    if (warp == 0) {
      // lane i holds column k0 + i of the diagonal block: L[k0 + j][k0 + i], j >= i
      double lcol[kPW];
#pragma unroll
      for (int j = 0; j < kPW; j++)
        lcol[j] = (lane < kb && j < kb && j >= lane) ? P.S[(size_t)(k0 + j) * n + k0 + lane] : 0.0;
      double yi = lane < kb ? x[k0 + lane] : 0.0;
#pragma unroll
      for (int j = kPW - 1; j >= 0; j--) {
        if (j < kb) {
          const double djj = __shfl_sync(0xffffffffu, lcol[j], j);
          const double xj = __shfl_sync(0xffffffffu, yi, j) / djj;
          if (lane == j) yi = xj;
          if (lane < j) yi -= lcol[j] * xj;
        }
      }
      if (lane < kb) x[k0 + lane] = yi;
    }
    __syncthreads();
    for (int r = tid; r < k0; r += nt) {
      double s = x[r];
      for (int j = 0; j < kb; j++) s -= P.S[(size_t)(k0 + j) * n + r] * x[k0 + j];
      x[r] = s;
    }
    __syncthreads();
  }
  // back-substitution: xV = V^-1 (-bV - sum W' xU) per point
  for (int p = tid; p < P.npv; p += nt) {
    double t[3] = {-P.bV[3 * (size_t)p], -P.bV[3 * (size_t)p + 1], -P.bV[3 * (size_t)p + 2]};
    for (int q = P.pt_ptr[p]; q < P.pt_ptr[p + 1]; q++) {
      const int e = P.p2e[q];
      const int ci = P.slot2int[P.e_cam[e]];
      if (ci < 0) continue;
      const double* We = P.W + (size_t)e * (BC * 3);
      const double* xu = x + (size_t)ci * BC;
#pragma unroll
      for (int i = 0; i < BC; i++) {
        t[0] -= We[i * 3] * xu[i];
        t[1] -= We[i * 3 + 1] * xu[i];
        t[2] -= We[i * 3 + 2] * xu[i];
      }
    }
    const double* Vi = P.Vinv + (size_t)p * 9;
#pragma unroll
    for (int i = 0; i < 3; i++) x[n + 3 * (size_t)p + i] = Vi[i * 3] * t[0] + Vi[i * 3 + 1] * t[1] + Vi[i * 3 + 2] * t[2];
  }
  __syncthreads();
  const bool ok = *flag == 0;
  if (!ok)  // SolverCholeskySchur.hpp:151-154
    for (int i = tid; i < n + 3 * P.npv; i += nt) x[i] = 0.0;
  __syncthreads();
  return ok;
}

template <int BC>
__device__ void oplus(const BProb& P) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int c = tid; c < P.ncv; c += nt) {
    double* s = P.cam + (size_t)P.cam_slot[c] * 16;
    const double* d = P.inc + (size_t)c * BC;
    double dR[9], R[9];
    so3_exp(d, dR);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) R[i * 3 + j] = dR[i * 3] * s[j] + dR[i * 3 + 1] * s[3 + j] + dR[i * 3 + 2] * s[6 + j];
#pragma unroll
    for (int i = 0; i < 9; i++) s[i] = R[i];
#pragma unroll
    for (int i = 0; i < 3; i++) s[9 + i] += d[3 + i];
    if (BC == 9)
#pragma unroll
      for (int i = 0; i < 3; i++) s[12 + i] += d[6 + i];
  }
  for (int i = tid; i < 3 * P.npv; i += nt) P.pt[i] += P.inc[P.n + i];
}

__device__ inline void copy_params(const BProb& P, bool to_backup) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const size_t nc = (size_t)P.nc_all * 16, np = (size_t)P.np_all * 3;
  double* cd = to_backup ? P.cam_bck : P.cam;
  const double* cs = to_backup ? P.cam : P.cam_bck;
  double* pd = to_backup ? P.pt_bck : P.pt;
  const double* ps = to_backup ? P.pt : P.pt_bck;
  for (size_t i = tid; i < nc; i += nt) cd[i] = cs[i];
  for (size_t i = tid; i < np; i += nt) pd[i] = ps[i];
}

template <int BC>
__device__ double max_abs_b(const BProb& P, double* sh) {
  const int nb = P.n, nv = 3 * P.npv;
  return cta_max(nb + nv, [&](int i) { return fabs(i < nb ? P.bU[i] : P.bV[i - nb]); }, sh);
}

template <int BC>
__device__ double max_abs_hdiag(const BProb& P, double* sh) {
  const int nb = P.n, nv = 3 * P.npv;
  return cta_max(
      nb + nv,
      [&](int i) {
        return fabs(i < nb ? P.U[(size_t)(i / BC) * BC * BC + (i % BC) * (BC + 1)] : P.V[(size_t)((i - nb) / 3) * 9 + ((i - nb) % 3) * 4]);
      },
      sh);
}

// The LM solve of one problem (nelson/LevenbergMarquardt.hpp:36-146; the
// decisions on thread 0, as lm_kernels.cuh orders them).
template <int BC>
__device__ void solve_problem(const BProb& P, const BSettings& s, BReport* rep, double* smem, LmS& st, double* sh,
                              int* flag) {
  const int tid = threadIdx.x;
  if (tid == 0) rep->t_start = global_ns();
  double c0 = cost<BC>(P, sh);
  jacobian_pass<BC>(P);
  __syncthreads();
  const double mb = max_abs_b<BC>(P, sh);
  if (tid == 0) {
    st.chi2 = st.oldChi2 = c0;
    st.maxAbsB = mb;
    st.done = 0;
    st.iter = -1;
    st.subiter = 0;
    st.nsub = 0;
    st.mu = 0.0;
    if (mb <= s.epsBVector) {
      st.done = 1;
      st.reason = NL_SUCCESS_AT_START;
    }
  }
  __syncthreads();
  if (!st.done) {
    copy_params(P, true);
    const double hd = max_abs_hdiag<BC>(P, sh);
    if (tid == 0) {
      st.mu = s.tau * hd;  // LevenbergMarquardt.hpp:58
      st.curV = s.initV;
      st.iter = 0;
      if (s.maxNumIt <= 0) {
        st.done = 1;
        st.reason = NL_MAX_ITERATION_REACHED;
      }
    }
    __syncthreads();
  }
  while (!st.done) {
    const bool ok = compute_increment<BC>(P, st.mu, smem, flag);
    const double mu = st.mu;
    const int nn = P.n + 3 * P.npv;
    const double a = cta_sum(nn, [&](int i) { return P.inc[i] * P.inc[i]; }, P.part, sh);
    const double den = cta_sum(
        nn,
        [&](int i) {
          const double x = P.inc[i], g = i < P.n ? P.bU[i] : P.bV[i - P.n];
          return x * (mu * x - g);
        },
        P.part, sh);
    if (tid == 0) {
      st.ok = ok && isfinite(a);
      st.incSq = st.ok ? a : 0.0;
      st.den = den;
      st.apply = 0;
      if (st.ok && st.iter >= s.minNumIt && st.incSq <= s.epsIncSquare) {  // LevenbergMarquardt.hpp:73-75
        st.done = 1;
        st.reason = NL_SUCCESS_SMALL_INCREMENT;
      } else {
        st.apply = st.ok;
      }
    }
    __syncthreads();
    if (st.done) break;
    double cn = 0.0;
    if (st.apply) {
      oplus<BC>(P);
      __syncthreads();
      cn = cost<BC>(P, sh);
    }
    if (tid == 0) {
      // LevenbergMarquardt.hpp:78-129
      double rho = -1.0;
      if (st.apply) {
        st.chi2_new = cn;
        rho = (st.oldChi2 - cn) / st.den;
      }
      st.rho = rho;
      st.acc = st.apply && rho > 0.0;
      st.nsub++;
      if (st.acc) {
        st.chi2 = cn;
        if (st.iter > s.minNumIt && st.maxAbsB <= s.epsBVector) {
          st.done = 1;
          st.reason = NL_SUCCESS_EPS_B;
        } else if (st.iter > s.minNumIt && cn < s.epsChi2) {
          st.done = 1;
          st.reason = NL_SUCCESS_SMALL_RESIDUALS;
        } else {
          const double fc = 2.0 * rho - 1.0;
          double alpha = fmin(s.maxScale, 1.0 - fc * fc * fc);
          alpha = fmax(s.minScale, alpha);
          st.mu = st.mu * alpha;
          st.curV = s.initV;
        }
      } else {
        st.mu = st.mu * st.curV;
        st.curV = st.curV * s.penaltyV;
      }
      if (!st.done) {
        st.subiter++;
        if (st.subiter >= s.maxNumSubIt) {
          st.done = 1;
          st.reason = NL_MAX_SUBITERATION_REACHED;
        }
      }
    }
    __syncthreads();
    if (!st.acc) {
      copy_params(P, false);  // rollbackSolution
      __syncthreads();
    }
    if (st.done) break;
    if (st.acc) {
      // update(true) at the accepted point, backupSolution
      const double c1 = cost<BC>(P, sh);
      jacobian_pass<BC>(P);
      __syncthreads();
      const double mb2 = max_abs_b<BC>(P, sh);
      copy_params(P, true);
      if (tid == 0) {
        st.chi2 = c1;
        st.oldChi2 = c1;
        st.maxAbsB = mb2;
        st.iter++;
        st.subiter = 0;
        if (st.iter >= s.maxNumIt) {
          st.done = 1;
          st.reason = NL_MAX_ITERATION_REACHED;
        }
      }
      __syncthreads();
    }
  }
  __syncthreads();
  if (tid == 0) {
    rep->reason = st.reason;
    rep->iterations = st.iter;
    rep->subiterations = st.nsub;
    rep->chi2 = st.chi2;
    rep->mu = st.mu;
    rep->t_end = global_ns();
  }
  __syncthreads();
}

template <int BC, int NT>
__global__ void __launch_bounds__(NT) batch_lm_kernel(const BProb* __restrict__ probs, const int* __restrict__ order,
                                                      int nprob, int* __restrict__ queue, BSettings s,
                                                      BReport* __restrict__ reps) {
  extern __shared__ __align__(16) double smem[];
  __shared__ BProb Ps;
  __shared__ LmS st;
  __shared__ double sh[40];
  __shared__ int q_s, flag;
  for (;;) {
    if (threadIdx.x == 0) q_s = atomicAdd(queue, 1);
    __syncthreads();
    const int q = q_s;
    if (q >= nprob) return;
    const int pi = order[q];
    if (threadIdx.x == 0) Ps = probs[pi];
    __syncthreads();
    solve_problem<BC>(Ps, s, reps + pi, smem, st, sh, &flag);
    __syncthreads();
  }
}

using BatchKernel = void (*)(const BProb*, const int*, int, int*, BSettings, BReport*);

template <int BC>
BatchKernel pick_kernel(int nt) {
  switch (nt) {
    case 128: return batch_lm_kernel<BC, 128>;
    case 256: return batch_lm_kernel<BC, 256>;
    default: return batch_lm_kernel<BC, 512>;
  }
}

}  // namespace
}  // namespace nl

// ===========================================================================
// Host side.
struct nl_batch {
  int n = 0, bc = 0, device = 0, max_n = 0;
  std::vector<nl_problem*> hs;
  nl::DevBuf arena, probs, order, queue, reps;
  std::vector<nl::BProb> hp;            // host copies of the descriptors
  std::vector<size_t> off_cam, off_pt;  // state offsets in the arena (doubles)
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int tuned_nt = 0, tuned_cps = 0;  // autotuner's choice (0: not tuned)
  float tune_ms[6] = {0, 0, 0, 0, 0, 0};
  ~nl_batch() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
  }
};

extern "C" {

nl_status nl_batch_create(nl_problem** hs, int n, nl_batch** out) {
  using namespace nl;
  if (!hs || n <= 0 || !out) return NL_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<nl_batch> b(new nl_batch());
  b->n = n;
  b->hs.assign(hs, hs + n);
  std::vector<nl_problem_view> vs(n);
  for (int i = 0; i < n; i++) {
    if (!hs[i]) return NL_ERR_ARG;
    for (int j = 0; j < i; j++)
      if (hs[j] == hs[i]) return NL_ERR_ARG;
    nl_status s = nl_problem_get_view(hs[i], &vs[i]);
    if (s != NL_OK) return s;
    if (!vs[i].ready) return NL_ERR_STATE;
    if (vs[i].bc != vs[0].bc) return NL_ERR_UNSUPPORTED;
    if ((long long)vs[i].ncv * vs[i].bc > kMaxN) return NL_ERR_UNSUPPORTED;
  }
  b->bc = vs[0].bc;
  const int bc = b->bc;
  int dev = 0;
  NL_CUDA(cudaGetDevice(&dev));
  b->device = dev;
  NL_CUDA(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
  NL_CUDA(cudaEventCreate(&b->e0));
  NL_CUDA(cudaEventCreate(&b->e1));
  // ---- host structure of every problem, then one arena for all of it ----
  struct HostProb {
    std::vector<int> e_cam, e_pt, cam_ptr, cam_slot, slot2int, pt_ptr, p2e, s_i, s_j, s_ptr, pa, pb;
    std::vector<double> e_obs, e_w;
  };
  std::vector<HostProb> H(n);
  std::vector<double> work(n, 0.0);
  size_t total = 0;  // bytes
  auto al = [](size_t x) { return (x + 255) / 256 * 256; };
  std::vector<std::vector<size_t>> offs(n);
  for (int i = 0; i < n; i++) {
    const nl_problem_view& v = vs[i];
    HostProb& h = H[i];
    const int ne = (int)v.e_cam->size(), ncv = v.ncv, npv = v.npv;
    const std::vector<int>& eo = *v.eorder;
    std::vector<int> epos(ne);
    for (int t = 0; t < ne; t++) epos[eo[t]] = t;
    h.e_cam.resize(ne);
    h.e_pt.resize(ne);
    h.e_obs.resize(2 * (size_t)ne);
    h.e_w.resize(ne);
    h.cam_ptr.assign(ncv + 1, 0);
    for (int t = 0; t < ne; t++) {
      const int e = eo[t];
      const bool cf = (*v.e_camfix)[e] != 0, pf = (*v.e_ptfix)[e] != 0;
      h.e_cam[t] = cf ? ncv + (*v.e_cam)[e] : (*v.e_cam)[e];
      h.e_pt[t] = pf ? npv + (*v.e_pt)[e] : (*v.e_pt)[e];
      h.e_obs[2 * t] = (*v.e_obs)[2 * (size_t)e];
      h.e_obs[2 * t + 1] = (*v.e_obs)[2 * (size_t)e + 1];
      h.e_w[t] = (*v.e_w)[e];
      if (!cf) h.cam_ptr[(*v.perm)[(*v.e_cam)[e]] + 1]++;
    }
    for (int c = 0; c < ncv; c++) h.cam_ptr[c + 1] += h.cam_ptr[c];
    h.cam_slot.resize(ncv);
    h.slot2int.assign(ncv + v.ncf, -1);
    for (int u = 0; u < ncv; u++) {
      h.cam_slot[(*v.perm)[u]] = u;
      h.slot2int[u] = (*v.perm)[u];
    }
    const std::vector<int>& po = *v.porder;
    h.p2e.resize(po.size());
    h.pt_ptr.assign(npv + 1, 0);
    for (size_t t = 0; t < po.size(); t++) {
      h.p2e[t] = epos[po[t]];
      h.pt_ptr[(*v.e_pt)[po[t]] + 1]++;
    }
    for (int p = 0; p < npv; p++) h.pt_ptr[p + 1] += h.pt_ptr[p];
    // S blocks (i <= j) and their pairs, points ascending (MatrixWWtMultiplier::prepare order)
    std::vector<int> bid((size_t)ncv * ncv, -1);
    for (int c = 0; c < ncv; c++) {
      bid[(size_t)c * ncv + c] = (int)h.s_i.size();
      h.s_i.push_back(c);
      h.s_j.push_back(c);
    }
    std::vector<std::vector<std::pair<int, int>>> blist;
    blist.resize(ncv);
    std::vector<int> ve;
    for (int p = 0; p < npv; p++) {
      ve.clear();
      for (int t = h.pt_ptr[p]; t < h.pt_ptr[p + 1]; t++)
        if (h.e_cam[h.p2e[t]] < ncv) ve.push_back(h.p2e[t]);
      for (int a : ve)
        for (int bb : ve) {
          const int ci = (*v.perm)[h.e_cam[a]], cj = (*v.perm)[h.e_cam[bb]];
          if (ci > cj) continue;
          int& id = bid[(size_t)ci * ncv + cj];
          if (id < 0) {
            id = (int)h.s_i.size();
            h.s_i.push_back(ci);
            h.s_j.push_back(cj);
            blist.emplace_back();
          }
          blist[id].push_back({a, bb});
        }
    }
    h.s_ptr.assign(h.s_i.size() + 1, 0);
    for (size_t q = 0; q < h.s_i.size(); q++) {
      h.s_ptr[q + 1] = h.s_ptr[q] + (int)blist[q].size();
      for (auto& pr : blist[q]) {
        h.pa.push_back(pr.first);
        h.pb.push_back(pr.second);
      }
    }
    const int nn = ncv * bc;
    work[i] = (double)h.pa.size() * bc * bc * 3 + (double)nn * nn * nn / 6.0 + 60.0 * ne * bc;
    // arena layout (bytes)
    const size_t nc_all = (size_t)ncv + v.ncf, np_all = (size_t)npv + v.npf;
    const size_t sizes[] = {
        sizeof(int) * ne, sizeof(int) * ne, sizeof(double) * 2 * ne, sizeof(double) * ne,                  // 0-3
        sizeof(int) * (ncv + 1), sizeof(int) * ncv, sizeof(int) * (ncv + v.ncf), sizeof(int) * (npv + 1),  // 4-7
        sizeof(int) * h.p2e.size(), sizeof(int) * h.s_i.size(), sizeof(int) * h.s_j.size(),                 // 8-10
        sizeof(int) * h.s_ptr.size(), sizeof(int) * h.pa.size(), sizeof(int) * h.pb.size(),                 // 11-13
        sizeof(double) * nc_all * 16, sizeof(double) * np_all * 3,                                          // 14-15
        sizeof(double) * nc_all * 16, sizeof(double) * np_all * 3,                                          // 16-17
        sizeof(double) * ne * bc * 3, sizeof(double) * ne * bc * 3,                                         // 18-19 W, Y
        sizeof(double) * ncv * bc * bc, sizeof(double) * ncv * bc,                                          // 20-21 U, bU
        sizeof(double) * npv * 9, sizeof(double) * npv * 9, sizeof(double) * npv * 3, sizeof(double) * npv * 3,  // 22-25
        sizeof(double) * nn * nn, sizeof(double) * nn, sizeof(double) * (nn + 3 * npv),                   // 26-28
        sizeof(double) * ((size_t)std::max(ne, nn + 3 * npv) / 32 + 64)};                                   // 29
    for (size_t s : sizes) {
      offs[i].push_back(total);
      total += al(std::max<size_t>(s, 8));
    }
    b->max_n = std::max(b->max_n, nn);
  }
  nl_status s;
  if ((s = b->arena.alloc(total)) != NL_OK) return s;
  char* base = static_cast<char*>(b->arena.p);
  b->hp.resize(n);
  b->off_cam.resize(n);
  b->off_pt.resize(n);
  for (int i = 0; i < n; i++) {
    const nl_problem_view& v = vs[i];
    HostProb& h = H[i];
    const std::vector<size_t>& o = offs[i];
    BProb& P = b->hp[i];
    P = BProb{};
    P.ncv = v.ncv;
    P.nc_all = v.ncv + v.ncf;
    P.npv = v.npv;
    P.np_all = v.npv + v.npf;
    P.ne = (int)h.e_cam.size();
    P.n = v.ncv * bc;
    P.nS = (int)h.s_i.size();
    P.f = v.f;
    P.cx = v.cx;
    P.cy = v.cy;
    auto put = [&](int k, const void* src, size_t bytes) -> nl_status {
      if (bytes) NL_CUDA(cudaMemcpyAsync(base + o[k], src, bytes, cudaMemcpyHostToDevice, b->st));
      return NL_OK;
    };
#define NL_PUT(k, vec)                                                                              \
  if ((s = put(k, vec.data(), vec.size() * sizeof(vec[0]))) != NL_OK) return s;
    NL_PUT(0, h.e_cam) NL_PUT(1, h.e_pt) NL_PUT(2, h.e_obs) NL_PUT(3, h.e_w) NL_PUT(4, h.cam_ptr)
    NL_PUT(5, h.cam_slot) NL_PUT(6, h.slot2int) NL_PUT(7, h.pt_ptr) NL_PUT(8, h.p2e) NL_PUT(9, h.s_i)
    NL_PUT(10, h.s_j) NL_PUT(11, h.s_ptr) NL_PUT(12, h.pa) NL_PUT(13, h.pb)
#undef NL_PUT
    P.e_cam = reinterpret_cast<const int*>(base + o[0]);
    P.e_pt = reinterpret_cast<const int*>(base + o[1]);
    P.e_obs = reinterpret_cast<const double*>(base + o[2]);
    P.e_w = reinterpret_cast<const double*>(base + o[3]);
    P.cam_ptr = reinterpret_cast<const int*>(base + o[4]);
    P.cam_slot = reinterpret_cast<const int*>(base + o[5]);
    P.slot2int = reinterpret_cast<const int*>(base + o[6]);
    P.pt_ptr = reinterpret_cast<const int*>(base + o[7]);
    P.p2e = reinterpret_cast<const int*>(base + o[8]);
    P.s_i = reinterpret_cast<const int*>(base + o[9]);
    P.s_j = reinterpret_cast<const int*>(base + o[10]);
    P.s_ptr = reinterpret_cast<const int*>(base + o[11]);
    P.pa = reinterpret_cast<const int*>(base + o[12]);
    P.pb = reinterpret_cast<const int*>(base + o[13]);
    double* d[16];
    for (int k = 14; k < 30; k++) d[k - 14] = reinterpret_cast<double*>(base + o[k]);
    P.cam = d[0];
    P.pt = d[1];
    P.cam_bck = d[2];
    P.pt_bck = d[3];
    P.W = d[4];
    P.Y = d[5];
    P.U = d[6];
    P.bU = d[7];
    P.V = d[8];
    P.Vinv = d[9];
    P.bV = d[10];
    P.xV0 = d[11];
    P.S = d[12];
    P.bS = d[13];
    P.inc = d[14];
    P.part = d[15];
    b->off_cam[i] = o[14];
    b->off_pt[i] = o[15];
  }
  // W / Y of edges without a variable camera or point are never read; zero all once
  if ((s = upload(b->probs, b->hp, b->st)) != NL_OK) return s;
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return work[x] > work[y]; });
  if ((s = upload(b->order, ord, b->st)) != NL_OK) return s;
  if ((s = b->queue.alloc(sizeof(int) * 8)) != NL_OK) return s;
  if ((s = b->reps.alloc(sizeof(BReport) * n)) != NL_OK) return s;
  NL_CUDA(cudaStreamSynchronize(b->st));
  *out = b.release();
  return NL_OK;
}

nl_status nl_batch_destroy(nl_batch* b) {
  if (!b) return NL_ERR_ARG;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->st);
  delete b;
  return NL_OK;
}

}  // extern "C"

namespace {

nl_status batch_launch(nl_batch* b, const nl::BSettings& s, int nt, int cps, float* ms) {
  using namespace nl;
  const size_t smem = sizeof(double) * (size_t)std::max(b->max_n, 1) * kPLd;
  BatchKernel k = b->bc == 9 ? pick_kernel<9>(nt) : pick_kernel<6>(nt);
  NL_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int sms = 0, occ = 0;
  NL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  NL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, nt, smem));
  if (occ <= 0) return NL_ERR_UNSUPPORTED;
  const int grid = std::max(1, std::min(b->n, sms * std::min(cps, occ)));
  NL_CUDA(cudaMemsetAsync(b->queue.p, 0, sizeof(int), b->st));
  NL_CUDA(cudaEventRecord(b->e0, b->st));
  k<<<grid, nt, smem, b->st>>>(b->probs.as<BProb>(), b->order.as<int>(), b->n, b->queue.as<int>(), s,
                               b->reps.as<BReport>());
  NL_CUDA(cudaGetLastError());
  NL_CUDA(cudaEventRecord(b->e1, b->st));
  NL_CUDA(cudaEventSynchronize(b->e1));
  NL_CUDA(cudaEventElapsedTime(ms, b->e0, b->e1));
  return NL_OK;
}

// parameters: handles <-> arena
nl_status batch_params(nl_batch* b, bool to_arena) {
  char* base = static_cast<char*>(b->arena.p);
  for (int i = 0; i < b->n; i++) {
    nl_problem_view v;
    nl_status s = nl_problem_get_view(b->hs[i], &v);
    if (s != NL_OK) return s;
    const size_t nc = (size_t)(v.ncv + v.ncf) * 16 * sizeof(double), np = (size_t)(v.npv + v.npf) * 3 * sizeof(double);
    double* ac = reinterpret_cast<double*>(base + b->off_cam[i]);
    double* ap = reinterpret_cast<double*>(base + b->off_pt[i]);
    if (to_arena) {
      NL_CUDA(cudaMemcpyAsync(ac, v.d_cam, nc, cudaMemcpyDeviceToDevice, b->st));
      if (np) NL_CUDA(cudaMemcpyAsync(ap, v.d_pt, np, cudaMemcpyDeviceToDevice, b->st));
    } else {
      NL_CUDA(cudaMemcpyAsync(v.d_cam, ac, nc, cudaMemcpyDeviceToDevice, b->st));
      if (np) NL_CUDA(cudaMemcpyAsync(v.d_pt, ap, np, cudaMemcpyDeviceToDevice, b->st));
    }
  }
  return NL_OK;
}

}  // namespace

extern "C" {

nl_status nl_batch_autotune(nl_batch* b, const nl_lm_settings* st, int* nt_out, int* cps_out) {
  using namespace nl;
  if (!b || !st) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(b->device));
  BSettings s{st->maxNumIt, st->maxNumSubIt, st->minNumIt, 0, st->epsBVector, st->epsIncSquare, st->epsChi2,
              st->tau, st->penaltyV, st->initV, st->maxScaleFactor, st->minScaleFactor};
  const int cand_nt[3] = {128, 256, 512};
  const int cand_cps[2] = {1, 2};
  float best = 1e30f;
  int bn = 256, bcps = 1, q = 0;
  for (int a = 0; a < 3; a++)
    for (int c = 0; c < 2; c++, q++) {
      nl_status r = batch_params(b, true);  // every candidate starts from the handles' parameters
      if (r != NL_OK) return r;
      float ms = 0;
      r = batch_launch(b, s, cand_nt[a], cand_cps[c], &ms);
      if (r == NL_ERR_UNSUPPORTED) {
        b->tune_ms[q] = -1;
        continue;
      }
      if (r != NL_OK) return r;
      b->tune_ms[q] = ms;
      if (ms < best) {
        best = ms;
        bn = cand_nt[a];
        bcps = cand_cps[c];
      }
    }
  b->tuned_nt = bn;
  b->tuned_cps = bcps;
  if (nt_out) *nt_out = bn;
  if (cps_out) *cps_out = bcps;
  return NL_OK;
}

nl_status nl_batch_lm_solve(nl_batch* b, const nl_lm_settings* st, int threads, int ctas_per_sm,
                            nl_solve_report* reps, double* latency_ms, double* device_ms) {
  using namespace nl;
  if (!b || !st) return NL_ERR_ARG;
  if (threads != 0 && threads != 128 && threads != 256 && threads != 512) return NL_ERR_ARG;
  if (ctas_per_sm < 0 || ctas_per_sm > 4) return NL_ERR_ARG;
  NL_CUDA(cudaSetDevice(b->device));
  BSettings s{st->maxNumIt, st->maxNumSubIt, st->minNumIt, 0, st->epsBVector, st->epsIncSquare, st->epsChi2,
              st->tau, st->penaltyV, st->initV, st->maxScaleFactor, st->minScaleFactor};
  const int nt = threads ? threads : (b->tuned_nt ? b->tuned_nt : 256);
  const int cps = ctas_per_sm ? ctas_per_sm : (b->tuned_cps ? b->tuned_cps : 1);
  nl_status r = batch_params(b, true);
  if (r != NL_OK) return r;
  float ms = 0;
  if ((r = batch_launch(b, s, nt, cps, &ms)) != NL_OK) return r;
  if ((r = batch_params(b, false)) != NL_OK) return r;
  std::vector<BReport> hr(b->n);
  NL_CUDA(cudaMemcpyAsync(hr.data(), b->reps.p, sizeof(BReport) * b->n, cudaMemcpyDeviceToHost, b->st));
  NL_CUDA(cudaStreamSynchronize(b->st));
  unsigned long long t0 = ~0ull;
  for (auto& x : hr) t0 = std::min(t0, x.t_start);
  for (int i = 0; i < b->n; i++) {
    if (reps) {
      reps[i].reason = hr[i].reason;
      reps[i].iterations = hr[i].iterations;
      reps[i].subiterations = hr[i].subiterations;
      reps[i].n_trace = 0;
      reps[i].chi2 = hr[i].chi2;
      reps[i].mu = hr[i].mu;
      reps[i].device_ms = 1e-6 * (double)(hr[i].t_end - hr[i].t_start);
    }
    if (latency_ms) latency_ms[i] = 1e-6 * (double)(hr[i].t_end - t0);
  }
  if (device_ms) *device_ms = ms;
  return NL_OK;
}

}  // extern "C"
