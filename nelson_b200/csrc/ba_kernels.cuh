// ba_kernels.cuh -- BA edge evaluation fused with the J'J / J'r accumulation.
//
// Replaces BaseSection::evaluateEdges + BaseSection::updateHessianBlocks
// (nelson/BaseSection.cpp:88-169, 5-86) for the projection EdgeBinaryUV of
// nelson/samples/BASchurPerfomances.cpp:195-232.  No float atomics: every
// Hessian block is produced by exactly one thread or one CTA, which sums its
// edges in a fixed order, so results are bit-reproducible run to run.
//
//   cost_kernel      one thread per edge, FP64 residual, chi2 per CTA, then
//                    cost_finalize sums the CTA partials in index order.
//   cam_pass_kernel  one CTA per (internal) camera: edges in W-UID order,
//                    writes each W block (J_c' J_p) and reduces U_c, bU_c.
//   pt_pass_kernel   one thread per point: V_p, bV_p.
#pragma once

#include <type_traits>

#include "nl_common.cuh"

namespace nl {

struct BaDev {
  int bc, nci, nc_all, np_var, np_all, ne, ngrp;
  double f_fixed, cx, cy;
  double* cam;      // nc_all x 16 camera state (R, t, f, k1, k2, pad)
  double* pt;       // np_all x 3
  // camera-major ("E-order") edges: W-UID order, fixed-point edges last per camera,
  // fixed-camera edges at the very end
  const int* e_cam;  // camera slot
  const int* e_pt;   // point slot
  const double* e_obs;
  const double* e_w;
  const int* cam_grp_ptr;   // nci + 1, groups of internal camera c
  const int* grp_edge_ptr;  // ngrp + 1, E-order edges of a group
  const int* grp_wuid;      // W uid of a group, -1 for a fixed point
  const int* cam_uid;       // internal camera -> U uid (-1: no block)
  const int* cam_slot;      // internal camera -> camera slot
  // point-major edges of variable points
  const int* pt_edge_ptr;   // np_var + 1
  const int* p_cam;         // camera slot
  const double* p_obs;
  const double* p_w;
  const int* pt_vuid;       // point -> V uid (-1: no block)
};

// Projection residual in FP64 and, optionally, the Jacobians in T.
//   P = R X + t, (x, y) = P.xy / P.z, d = 1 + k1 r^2 + k2 r^4,
//   pixel = f d (x, y) + (cx, cy), r = pixel - z.
// Camera tangent [dw, dt (, df, dk1, dk2)] with R <- exp(dw) R.
template <typename T, int BC, bool JC, bool JP>
__device__ __forceinline__ void ba_project(const double* __restrict__ cs, const double* __restrict__ X,
                                           double z0, double z1, double f_fixed, double cx, double cy,
                                           double& r0, double& r1, T* Jc, T* Jp) {
  const double a0 = cs[0] * X[0] + cs[1] * X[1] + cs[2] * X[2];
  const double a1 = cs[3] * X[0] + cs[4] * X[1] + cs[5] * X[2];
  const double a2 = cs[6] * X[0] + cs[7] * X[1] + cs[8] * X[2];
  const double P0 = a0 + cs[9], P1 = a1 + cs[10], P2 = a2 + cs[11];
  const double iz = 1.0 / P2;
  const double x = P0 * iz, y = P1 * iz;
  double f, k1, k2;
  if (BC == 9) {
    f = cs[12];
    k1 = cs[13];
    k2 = cs[14];
  } else {
    f = f_fixed;
    k1 = 0.0;
    k2 = 0.0;
  }
  const double r2 = x * x + y * y;
  const double d = 1.0 + r2 * (k1 + k2 * r2);
  r0 = f * d * x + cx - z0;
  r1 = f * d * y + cy - z1;
  if (!JC && !JP) return;
  const double g = 2.0 * (k1 + 2.0 * k2 * r2);
  const double m00 = f * (d + g * x * x), m01 = f * g * x * y, m11 = f * (d + g * y * y);
  double M[6];
  M[0] = m00 * iz;
  M[1] = m01 * iz;
  M[2] = -(m00 * x + m01 * y) * iz;
  M[3] = m01 * iz;
  M[4] = m11 * iz;
  M[5] = -(m01 * x + m11 * y) * iz;
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const double* m = M + 3 * i;
    if (JP) {
#pragma unroll
      for (int j = 0; j < 3; j++) Jp[i * 3 + j] = (T)(m[0] * cs[j] + m[1] * cs[3 + j] + m[2] * cs[6 + j]);
    }
    if (JC) {
      T* jc = Jc + i * BC;
      jc[0] = (T)(-m[1] * a2 + m[2] * a1);
      jc[1] = (T)(m[0] * a2 - m[2] * a0);
      jc[2] = (T)(-m[0] * a1 + m[1] * a0);
      jc[3] = (T)m[0];
      jc[4] = (T)m[1];
      jc[5] = (T)m[2];
    }
  }
  if (JC && BC == 9) {
    Jc[6] = (T)(d * x);
    Jc[7] = (T)(f * x * r2);
    Jc[8] = (T)(f * x * r2 * r2);
    Jc[BC + 6] = (T)(d * y);
    Jc[BC + 7] = (T)(f * y * r2);
    Jc[BC + 8] = (T)(f * y * r2 * r2);
  }
}

// ---------------------------------------------------------------------------
// chi2 = sum_e w_e |r_e|^2 in FP64.  `active` (may be null) skips the launch
// body when the device-side LM state says so.
template <int BC, int NT>
static __global__ void __launch_bounds__(NT) cost_kernel(BaDev d, double* __restrict__ partial,
                                                  const int* __restrict__ active) {
  __shared__ double sh[NT / 32];
  if (active && !*active) return;
  double acc = 0.0;
  for (int e = blockIdx.x * NT + threadIdx.x; e < d.ne; e += gridDim.x * NT) {
    const double* cs = d.cam + (size_t)__ldg(d.e_cam + e) * 16;
    const double* X = d.pt + (size_t)__ldg(d.e_pt + e) * 3;
    double r0, r1;
    ba_project<double, BC, false, false>(cs, X, __ldg(d.e_obs + 2 * e), __ldg(d.e_obs + 2 * e + 1),
                                         d.f_fixed, d.cx, d.cy, r0, r1, nullptr, nullptr);
    acc += __ldg(d.e_w + e) * (r0 * r0 + r1 * r1);
  }
  const double s = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Sums the per-CTA partials in index order (deterministic) into *out.
template <int NT>
static __global__ void __launch_bounds__(NT) sum_partials_kernel(const double* __restrict__ partial, int n,
                                                          double* __restrict__ out,
                                                          const int* __restrict__ active) {
  __shared__ double sh[NT / 32];
  if (active && !*active) return;
  // each thread sums a contiguous chunk so the order is fixed for a given n
  const int per = (n + NT - 1) / NT;
  double acc = 0.0;
  const int b = threadIdx.x * per;
  for (int i = b; i < min(n, b + per); i++) acc += partial[i];
  const double s = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------
// Camera-major pass: U_c = sum w Jc'Jc, bU_c = sum w Jc'r, W_{c,p} = sum w Jc'Jp.
template <typename T, int BC, int NT>
static __global__ void __launch_bounds__(NT) cam_pass_kernel(BaDev d, T* __restrict__ U, T* __restrict__ W,
                                                      T* __restrict__ bU, const int* __restrict__ active) {
  constexpr int NU = BC * (BC + 1) / 2;  // upper triangle of U_c
  constexpr int NA = NU + BC;            // + bU_c
  constexpr int LW = Layout<T, BC>::W;
  constexpr int LU = Layout<T, BC>::U;
  __shared__ double cs[16];
  __shared__ T red[NT / 32][NA];
  if (active && !*active) return;
  const int c = blockIdx.x;
  const int slot = d.cam_slot[c];
  if (threadIdx.x < 16) cs[threadIdx.x] = d.cam[(size_t)slot * 16 + threadIdx.x];
  __syncthreads();
  T acc[NA];
#pragma unroll
  for (int i = 0; i < NA; i++) acc[i] = (T)0;
  const int g0 = d.cam_grp_ptr[c], g1 = d.cam_grp_ptr[c + 1];
  for (int g = g0 + threadIdx.x; g < g1; g += NT) {
    T wacc[BC * 3];
#pragma unroll
    for (int i = 0; i < BC * 3; i++) wacc[i] = (T)0;
    const int wuid = d.grp_wuid[g];
    for (int e = d.grp_edge_ptr[g]; e < d.grp_edge_ptr[g + 1]; e++) {
      const double* X = d.pt + (size_t)d.e_pt[e] * 3;
      double r0, r1;
      T Jc[2 * BC], Jp[6];
      ba_project<T, BC, true, true>(cs, X, d.e_obs[2 * e], d.e_obs[2 * e + 1], d.f_fixed, d.cx, d.cy, r0,
                                    r1, Jc, Jp);
      const T w = (T)d.e_w[e];
      const T wr0 = w * (T)r0, wr1 = w * (T)r1;
      int q = 0;
#pragma unroll
      for (int i = 0; i < BC; i++) {
        const T wi0 = w * Jc[i], wi1 = w * Jc[BC + i];
#pragma unroll
        for (int j = i; j < BC; j++) acc[q++] += wi0 * Jc[j] + wi1 * Jc[BC + j];
      }
#pragma unroll
      for (int i = 0; i < BC; i++) acc[NU + i] += Jc[i] * wr0 + Jc[BC + i] * wr1;
      if (wuid >= 0) {
#pragma unroll
        for (int i = 0; i < BC; i++) {
          const T wi0 = w * Jc[i], wi1 = w * Jc[BC + i];
#pragma unroll
          for (int j = 0; j < 3; j++) wacc[i * 3 + j] += wi0 * Jp[j] + wi1 * Jp[3 + j];
        }
      }
    }
    if (wuid >= 0) {
      // 16-byte vector stores of the padded block
      using V16 = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
      constexpr int EPV = 16 / (int)sizeof(T);
      __align__(16) T blk[LW];
#pragma unroll
      for (int i = 0; i < LW; i++) blk[i] = i < BC * 3 ? wacc[i] : (T)0;
#pragma unroll
      for (int i = 0; i < LW / EPV; i++)
        reinterpret_cast<V16*>(W + (size_t)wuid * LW)[i] = reinterpret_cast<const V16*>(blk)[i];
    }
  }
  // deterministic CTA reduction: warp shuffles, then warps in index order
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NA; i++) {
    T v = warp_sum(acc[i]);
    if (lane == 0) red[warp][i] = v;
  }
  __syncthreads();
  const int uid = d.cam_uid[c];
  for (int i = threadIdx.x; i < NA; i += NT) {
    T s = (T)0;
#pragma unroll
    for (int w = 0; w < NT / 32; w++) s += red[w][i];
    if (i < NU) {
      if (uid >= 0) {
        // map packed-upper index i -> (r, cc)
        int r = 0, rem = i;
        while (rem >= BC - r) {
          rem -= BC - r;
          r++;
        }
        const int cc = r + rem;
        U[(size_t)uid * LU + r * BC + cc] = s;
        U[(size_t)uid * LU + cc * BC + r] = s;
      }
    } else {
      bU[(size_t)c * BC + (i - NU)] = s;
    }
  }
}

// ---------------------------------------------------------------------------
// Point-major pass: V_p = sum w Jp'Jp, bV_p = sum w Jp'r.
template <typename T, int BC, int NT>
static __global__ void __launch_bounds__(NT) pt_pass_kernel(BaDev d, T* __restrict__ V, T* __restrict__ bV,
                                                     const int* __restrict__ active) {
  constexpr int LV = Layout<T, BC>::V;
  if (active && !*active) return;
  const int p = blockIdx.x * NT + threadIdx.x;
  if (p >= d.np_var) return;
  const double X[3] = {d.pt[3 * (size_t)p], d.pt[3 * (size_t)p + 1], d.pt[3 * (size_t)p + 2]};
  T v[6] = {0, 0, 0, 0, 0, 0}, b[3] = {0, 0, 0};
  for (int e = d.pt_edge_ptr[p]; e < d.pt_edge_ptr[p + 1]; e++) {
    const double* cs = d.cam + (size_t)__ldg(d.p_cam + e) * 16;
    double r0, r1;
    T Jp[6];
    ba_project<T, BC, false, true>(cs, X, __ldg(d.p_obs + 2 * e), __ldg(d.p_obs + 2 * e + 1), d.f_fixed, d.cx,
                                   d.cy, r0, r1, nullptr, Jp);
    const T w = (T)__ldg(d.p_w + e);
    const T wr0 = w * (T)r0, wr1 = w * (T)r1;
    v[0] += w * (Jp[0] * Jp[0] + Jp[3] * Jp[3]);
    v[1] += w * (Jp[0] * Jp[1] + Jp[3] * Jp[4]);
    v[2] += w * (Jp[0] * Jp[2] + Jp[3] * Jp[5]);
    v[3] += w * (Jp[1] * Jp[1] + Jp[4] * Jp[4]);
    v[4] += w * (Jp[1] * Jp[2] + Jp[4] * Jp[5]);
    v[5] += w * (Jp[2] * Jp[2] + Jp[5] * Jp[5]);
    b[0] += Jp[0] * wr0 + Jp[3] * wr1;
    b[1] += Jp[1] * wr0 + Jp[4] * wr1;
    b[2] += Jp[2] * wr0 + Jp[5] * wr1;
  }
  const int uid = d.pt_vuid[p];
  if (uid >= 0) {
    T* o = V + (size_t)uid * LV;
    o[0] = v[0]; o[1] = v[1]; o[2] = v[2];
    o[3] = v[1]; o[4] = v[3]; o[5] = v[4];
    o[6] = v[2]; o[7] = v[4]; o[8] = v[5];
  }
  bV[3 * (size_t)p] = b[0];
  bV[3 * (size_t)p + 1] = b[1];
  bV[3 * (size_t)p + 2] = b[2];
}

// ---------------------------------------------------------------------------
// Problem::oplus on the device: cameras R <- exp(dw) R, t += dt (, f/k += d);
// points += d.  The camera increment is read at its internal position.
template <int BC>
static __global__ void oplus_cam_kernel(double* __restrict__ cam, const int* __restrict__ cam_slot_of_internal,
                                 int nci, const double* __restrict__ incU, const int* __restrict__ active) {
  if (active && !*active) return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nci) return;
  double* s = cam + (size_t)cam_slot_of_internal[c] * 16;
  const double* dlt = incU + (size_t)c * BC;
  double dR[9], R[9];
  so3_exp(dlt, dR);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) R[i * 3 + j] = dR[i * 3] * s[j] + dR[i * 3 + 1] * s[3 + j] + dR[i * 3 + 2] * s[6 + j];
#pragma unroll
  for (int i = 0; i < 9; i++) s[i] = R[i];
#pragma unroll
  for (int i = 0; i < 3; i++) s[9 + i] += dlt[3 + i];
  if (BC == 9) {
#pragma unroll
    for (int i = 0; i < 3; i++) s[12 + i] += dlt[6 + i];
  }
}

static __global__ void oplus_pt_kernel(double* __restrict__ pt, int np_var, const double* __restrict__ incV,
                                const int* __restrict__ active) {
  if (active && !*active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * np_var) return;
  pt[i] += incV[i];
}

}  // namespace nl

namespace nl {

// ---------------------------------------------------------------------------
// Parameter exchange with the caller: axis-angle cameras <-> stored state,
// and observation reordering into the device edge orders.  Done on the
// device so host buffers (pinned or not) are copied once, unchanged.
__device__ inline void so3_log_dev(const double* R, double* w) {
  const double tr = R[0] + R[4] + R[8];
  const double c = fmin(1.0, fmax(-1.0, 0.5 * (tr - 1.0)));
  const double th = acos(c);
  const double v0 = R[7] - R[5], v1 = R[2] - R[6], v2 = R[3] - R[1];
  if (th < 1e-4) {
    const double f = 0.5 * (1.0 + th * th / 6.0);
    w[0] = f * v0;
    w[1] = f * v1;
    w[2] = f * v2;
    return;
  }
  if (3.141592653589793 - th < 1e-4) {
    int k = 0;
    if (R[4] > R[k * 4]) k = 1;
    if (R[8] > R[k * 4]) k = 2;
    double a[3];
    const double d = sqrt(fmax(0.0, 0.5 * (R[k * 4] + 1.0)));
    for (int i = 0; i < 3; i++) a[i] = (i == k) ? d : (0.25 * (R[i * 3 + k] + R[k * 3 + i])) / d;
    const double nn = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    const double s = (v0 * a[0] + v1 * a[1] + v2 * a[2]) < 0 ? -1.0 : 1.0;
    for (int i = 0; i < 3; i++) w[i] = s * th * a[i] / nn;
    return;
  }
  const double f = th / (2.0 * sin(th));
  w[0] = f * v0;
  w[1] = f * v1;
  w[2] = f * v2;
}

static __global__ void cams_in_kernel(const double* __restrict__ in, double* __restrict__ state, int n, int bc,
                                      double f_fixed) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const double* a = in + (size_t)c * bc;
  double* s = state + (size_t)c * 16;
  double R[9];
  so3_exp(a, R);
  for (int i = 0; i < 9; i++) s[i] = R[i];
  s[9] = a[3];
  s[10] = a[4];
  s[11] = a[5];
  if (bc == 9) {
    s[12] = a[6];
    s[13] = a[7];
    s[14] = a[8];
  } else {
    s[12] = f_fixed;
    s[13] = 0.0;
    s[14] = 0.0;
  }
  s[15] = 0.0;
}

static __global__ void cams_out_kernel(const double* __restrict__ state, double* __restrict__ out, int n, int bc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const double* s = state + (size_t)c * 16;
  double* o = out + (size_t)c * bc;
  double w[3];
  so3_log_dev(s, w);
  o[0] = w[0];
  o[1] = w[1];
  o[2] = w[2];
  o[3] = s[9];
  o[4] = s[10];
  o[5] = s[11];
  if (bc == 9) {
    o[6] = s[12];
    o[7] = s[13];
    o[8] = s[14];
  }
}

// dst[t] = src[order[t]] for observations (2 doubles) and weights.
static __global__ void gather_obs_kernel(const double* __restrict__ obs, const double* __restrict__ w,
                                         const int* __restrict__ order, int n, double* __restrict__ dobs,
                                         double* __restrict__ dw) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int e = order[t];
  dobs[2 * (size_t)t] = obs[2 * (size_t)e];
  dobs[2 * (size_t)t + 1] = obs[2 * (size_t)e + 1];
  if (w) dw[t] = w[e];
}

}  // namespace nl
