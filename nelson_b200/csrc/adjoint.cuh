// adjoint.cuh -- implicit-function adjoint of a converged BA solve.
//
// At a converged solution x* the local gradient b(x, z, w) = sum_e w_e J_e' r_e
// vanishes.  For a loss L(x*) the implicit-function theorem gives
//     dL/dtheta = -mu' db/dtheta,   H mu = dL/dx,   H = db/dx,
// where H is the exact Hessian of the cost in the tangent coordinates of the
// parameters (Gauss-Newton part J'WJ plus the second-order terms
// sum w r d2r; at b = 0 the derivative of the local gradient along the
// retraction is that Hessian).  Per edge (r = pi(x) - z):
//     dL/dz_e = w_e J_e mu_e,     dL/dw_e = -(J_e mu_e) . r_e.
// The kernels here compute H v exactly in FP64 by forward-mode dual numbers
// through the projection and its Jacobian (hv_cam_kernel / hv_pt_kernel), and
// the per-edge VJP (vjp_edge_kernel).  mu is found by iterative refinement
// that reuses the Schur factorisation of J'WJ as the preconditioner.
// Camera tangent [dw, dt (, df, dk1, dk2)] with R <- exp(dw) R, as everywhere.
#pragma once

#include "ba_kernels.cuh"
#include "nl_common.cuh"

namespace nl {

struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.v * b.d + a.d * b.v}; }
__device__ __forceinline__ Dual operator*(double s, Dual a) { return {s * a.v, s * a.d}; }
__device__ __forceinline__ Dual operator+(Dual a, double s) { return {a.v + s, a.d}; }
__device__ __forceinline__ Dual dual_inv(Dual a) {
  const double i = 1.0 / a.v;
  return {i, -a.d * i * i};
}

// Projection, residual and both Jacobians in dual arithmetic (the same
// formulas as ba_project).
template <int BC>
__device__ __forceinline__ void proj_jac_dual(const Dual* R, const Dual* t, Dual f, Dual k1, Dual k2, const Dual* X,
                                              double z0, double z1, double cx, double cy, Dual* r, Dual* Jc,
                                              Dual* Jp) {
  const Dual a0 = R[0] * X[0] + R[1] * X[1] + R[2] * X[2];
  const Dual a1 = R[3] * X[0] + R[4] * X[1] + R[5] * X[2];
  const Dual a2 = R[6] * X[0] + R[7] * X[1] + R[8] * X[2];
  const Dual P0 = a0 + t[0], P1 = a1 + t[1], P2 = a2 + t[2];
  const Dual iz = dual_inv(P2);
  const Dual x = P0 * iz, y = P1 * iz;
  const Dual r2 = x * x + y * y;
  const Dual dd = (r2 * (k1 + k2 * r2)) + 1.0;
  r[0] = f * dd * x + (cx - z0);
  r[1] = f * dd * y + (cy - z1);
  const Dual g = 2.0 * (k1 + 2.0 * (k2 * r2));
  const Dual m00 = f * (dd + g * x * x), m01 = f * (g * x * y), m11 = f * (dd + g * y * y);
  Dual M[6];
  M[0] = m00 * iz;
  M[1] = m01 * iz;
  M[2] = -((m00 * x + m01 * y) * iz);
  M[3] = m01 * iz;
  M[4] = m11 * iz;
  M[5] = -((m01 * x + m11 * y) * iz);
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const Dual* m = M + 3 * i;
#pragma unroll
    for (int j = 0; j < 3; j++) Jp[i * 3 + j] = m[0] * R[j] + m[1] * R[3 + j] + m[2] * R[6 + j];
    Dual* jc = Jc + i * BC;
    jc[0] = m[2] * a1 - m[1] * a2;
    jc[1] = m[0] * a2 - m[2] * a0;
    jc[2] = m[1] * a0 - m[0] * a1;
    jc[3] = m[0];
    jc[4] = m[1];
    jc[5] = m[2];
  }
  if (BC == 9) {
    Jc[6] = dd * x;
    Jc[7] = f * x * r2;
    Jc[8] = f * x * r2 * r2;
    Jc[BC + 6] = dd * y;
    Jc[BC + 7] = f * y * r2;
    Jc[BC + 8] = f * y * r2 * r2;
  }
}

// Dual parameters of an edge: value at x*, derivative along v (vc: camera
// tangent direction or null for a fixed camera, vp: point direction or null).
template <int BC>
__device__ __forceinline__ void load_dual(const double* cs, const double* Xs, const double* vc, const double* vp,
                                          double f_fixed, Dual* R, Dual* t, Dual& f, Dual& k1, Dual& k2, Dual* X) {
  // d/de exp(e [w]x) R = [w]x R
  double w0 = 0, w1 = 0, w2 = 0;
  if (vc) {
    w0 = vc[0];
    w1 = vc[1];
    w2 = vc[2];
  }
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const double c0 = cs[j], c1 = cs[3 + j], c2 = cs[6 + j];
    R[j] = {c0, -w2 * c1 + w1 * c2};
    R[3 + j] = {c1, w2 * c0 - w0 * c2};
    R[6 + j] = {c2, -w1 * c0 + w0 * c1};
  }
#pragma unroll
  for (int i = 0; i < 3; i++) t[i] = {cs[9 + i], vc ? vc[3 + i] : 0.0};
  if (BC == 9) {
    f = {cs[12], vc ? vc[6] : 0.0};
    k1 = {cs[13], vc ? vc[7] : 0.0};
    k2 = {cs[14], vc ? vc[8] : 0.0};
  } else {
    f = {f_fixed, 0.0};
    k1 = {0.0, 0.0};
    k2 = {0.0, 0.0};
  }
#pragma unroll
  for (int i = 0; i < 3; i++) X[i] = {Xs[i], vp ? vp[i] : 0.0};
}

// (H v) for the cameras: one CTA per internal camera over its E-order edges.
// vU: internal camera order (BC per camera), vV: variable points (3 each).
// MODE: kHvFull the exact Hessian; kHvGN the Gauss-Newton part J'WJ v only
// (the dual part of r is J v; the terms with the dual part of J are the
// second-order ones); kGrad the gradient J'W r itself (v unused, may be null).
constexpr int kHvFull = 0, kHvGN = 1, kGrad = 2;
template <int MODE>
__device__ __forceinline__ double hv_term(double w, Dual j0, Dual j1, Dual r0, Dual r1) {
  if (MODE == kGrad) return w * (j0.v * r0.v + j1.v * r1.v);
  if (MODE == kHvGN) return w * (j0.v * r0.d + j1.v * r1.d);
  return w * (j0.d * r0.v + j0.v * r0.d + j1.d * r1.v + j1.v * r1.d);
}

template <int BC, int NT, int MODE = kHvFull>
static __global__ void __launch_bounds__(NT) hv_cam_kernel(BaDev d, const double* __restrict__ vU,
                                                           const double* __restrict__ vV, double* __restrict__ outU) {
  __shared__ double sh[NT / 32];
  __shared__ double cs[16];
  const int c = blockIdx.x;
  const int slot = d.cam_slot[c];
  if (threadIdx.x < 16) cs[threadIdx.x] = d.cam[(size_t)slot * 16 + threadIdx.x];
  __syncthreads();
  const double* vc = vU ? vU + (size_t)c * BC : nullptr;
  double acc[BC];
#pragma unroll
  for (int i = 0; i < BC; i++) acc[i] = 0.0;
  const int e0 = d.grp_edge_ptr[d.cam_grp_ptr[c]], e1 = d.grp_edge_ptr[d.cam_grp_ptr[c + 1]];
  for (int e = e0 + threadIdx.x; e < e1; e += NT) {
    const int ps = d.e_pt[e];
    Dual R[9], t[3], f, k1, k2, X[3], r[2], Jc[2 * BC], Jp[6];
    load_dual<BC>(cs, d.pt + (size_t)ps * 3, vc, (vV && ps < d.np_var) ? vV + (size_t)ps * 3 : nullptr, d.f_fixed,
                  R, t, f, k1, k2, X);
    proj_jac_dual<BC>(R, t, f, k1, k2, X, d.e_obs[2 * e], d.e_obs[2 * e + 1], d.cx, d.cy, r, Jc, Jp);
    const double w = d.e_w[e];
#pragma unroll
    for (int i = 0; i < BC; i++) acc[i] += hv_term<MODE>(w, Jc[i], Jc[BC + i], r[0], r[1]);
  }
#pragma unroll
  for (int i = 0; i < BC; i++) {
    const double s = block_sum<NT>(acc[i], sh);
    if (threadIdx.x == 0) outU[(size_t)c * BC + i] = s;
  }
}

// (H v) for the variable points: one thread per point over its P-order edges.
// slot2int: camera slot -> internal camera (-1 for a fixed camera).
template <int BC, int MODE = kHvFull>
static __global__ void hv_pt_kernel(BaDev d, const int* __restrict__ slot2int, const double* __restrict__ vU,
                                    const double* __restrict__ vV, double* __restrict__ outV) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.np_var) return;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int e = d.pt_edge_ptr[p]; e < d.pt_edge_ptr[p + 1]; e++) {
    const int cslot = d.p_cam[e];
    const int ci = slot2int[cslot];
    Dual R[9], t[3], f, k1, k2, X[3], r[2], Jc[2 * BC], Jp[6];
    load_dual<BC>(d.cam + (size_t)cslot * 16, d.pt + (size_t)p * 3, (vU && ci >= 0) ? vU + (size_t)ci * BC : nullptr,
                  vV ? vV + (size_t)p * 3 : nullptr, d.f_fixed, R, t, f, k1, k2, X);
    proj_jac_dual<BC>(R, t, f, k1, k2, X, d.p_obs[2 * e], d.p_obs[2 * e + 1], d.cx, d.cy, r, Jc, Jp);
    const double w = d.p_w[e];
#pragma unroll
    for (int j = 0; j < 3; j++) acc[j] += hv_term<MODE>(w, Jp[j], Jp[3 + j], r[0], r[1]);
  }
#pragma unroll
  for (int j = 0; j < 3; j++) outV[3 * (size_t)p + j] = acc[j];
}

// Per-edge VJP: with u = J_e mu_e, dL/dz_e = w_e u and dL/dw_e = -u . r_e,
// written at the edge's insertion index.
template <int BC>
static __global__ void vjp_edge_kernel(BaDev d, const int* __restrict__ eorder, const int* __restrict__ slot2int,
                                       const double* __restrict__ muU, const double* __restrict__ muV,
                                       double* __restrict__ g_obs, double* __restrict__ g_w) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.ne) return;
  const int cslot = d.e_cam[e], ps = d.e_pt[e];
  const int ci = slot2int[cslot];
  double r0, r1, Jc[2 * BC], Jp[6];
  ba_project<double, BC, true, true>(d.cam + (size_t)cslot * 16, d.pt + (size_t)ps * 3, d.e_obs[2 * e],
                                     d.e_obs[2 * e + 1], d.f_fixed, d.cx, d.cy, r0, r1, Jc, Jp);
  double u0 = 0.0, u1 = 0.0;
  if (ci >= 0) {
    const double* m = muU + (size_t)ci * BC;
#pragma unroll
    for (int i = 0; i < BC; i++) {
      u0 += Jc[i] * m[i];
      u1 += Jc[BC + i] * m[i];
    }
  }
  if (ps < d.np_var) {
    const double* m = muV + (size_t)ps * 3;
#pragma unroll
    for (int j = 0; j < 3; j++) {
      u0 += Jp[j] * m[j];
      u1 += Jp[3 + j] * m[j];
    }
  }
  const double w = d.e_w[e];
  const int u = eorder[e];
  g_obs[2 * (size_t)u] = w * u0;
  g_obs[2 * (size_t)u + 1] = w * u1;
  if (g_w) g_w[u] = -(u0 * r0 + u1 * r1);
}

// b := -rhs in the working precision of the Hessian (the Schur pipeline
// solves (J'WJ) x = -b).
template <typename T>
static __global__ void neg_to_b_kernel(const double* __restrict__ rhs, int n, T* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (T)(-rhs[i]);
}

// mu += inc; res = g - H mu is formed by resid_kernel after the H v pass.
static __global__ void acc_kernel(double* __restrict__ mu, const double* __restrict__ inc, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) mu[i] += inc[i];
}

// res = a - hv - mu v (the residual of (J'WJ + mu I) v = a; mu on the device)
static __global__ void damped_resid_kernel(const double* __restrict__ a, const double* __restrict__ hv,
                                           const double* __restrict__ v, const double* __restrict__ mu, int n,
                                           double* __restrict__ res) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) res[i] = a[i] - hv[i] - *mu * v[i];
}

// res = -g - hv - mu v (the residual of the LM step (J'WJ + mu I) v = -g)
static __global__ void step_resid_kernel(const double* __restrict__ g, const double* __restrict__ hv,
                                         const double* __restrict__ v, const double* __restrict__ mu, int n,
                                         double* __restrict__ res) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) res[i] = -g[i] - hv[i] - *mu * v[i];
}

static __global__ void resid_kernel(const double* __restrict__ g, const double* __restrict__ hv, int n,
                                    double* __restrict__ res) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) res[i] = g[i] - hv[i];
}

}  // namespace nl
