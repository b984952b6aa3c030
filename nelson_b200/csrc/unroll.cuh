// unroll.cuh -- reverse-mode differentiation through K recorded LM steps.
//
// The unrolled map: K accepted LevenbergMarquardt steps from x_0,
//     x_{k+1} = x_k (+) delta_k,   delta_k = -(J'WJ(x_k) + mu_k I)^-1 b(x_k),
// with b = sum_e w_e J_e' r_e and the damping schedule mu_k of the accepted
// steps held fixed (nelson/LevenbergMarquardt.hpp:63-141: computeIncrement(H,
// b, 0, mu) then oplus; the accept / reject decisions and the mu updates are
// discrete and are not differentiated).  (+) is the retraction R <- exp(dw) R,
// t += dt, intrinsics and points additive.
//
// With the adjoint lam_{k+1} of x_{k+1} in the tangent at x_{k+1}:
//   * through (+): the increment's adjoint is a = [J_l(dw)' lam_w, lam_rest]
//     (J_l the left Jacobian of SO(3): exp(dw + e) = exp(J_l(dw) e) exp(dw)),
//     and x_k's direct part is [exp(dw)' lam_w, lam_rest] (exp(dw) exp(e)
//     exp(-dw) = exp(exp(dw) e));
//   * through delta_k: with u = A^-1 a (A = J'WJ + mu I, symmetric, solved with
//     the Schur factorisation of the step), a' d delta = -u'(db + dA delta), so
//     every input theta receives -d/dtheta [psi + phi] with u, delta fixed,
//         psi = u' b = sum_e w_e (J_e u_e) . r_e,
//         phi = u' J'WJ delta = sum_e w_e (J_e u_e) . (J_e delta_e);
//     for an observation dL/dz_e += w_e J_e u_e, for a weight
//     dL/dw_e -= (J_e u_e) . (r_e + J_e delta_e), and for the parameters the
//     gradient of psi + phi along each tangent direction of x_k, taken by
//     forward-mode dual numbers through the projection and its Jacobian (the
//     Jacobian of x_k (+) e is the one at the perturbed point, as in the step).
// Every sum runs in a fixed order (one CTA per camera over its edges, one
// thread per point over its edges), so the result is reproducible.
#pragma once

#include "adjoint.cuh"
#include "ba_kernels.cuh"
#include "nl_common.cuh"

namespace nl {

// J_l(p) = I + (1 - cos t) / t^2 [p]x + (t - sin t) / t^3 [p]x^2, t = |p|.
__device__ inline void so3_left_jacobian(const double* p, double* J) {
  const double t2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
  double A, B;
  if (t2 < 1e-6) {  // series; the next terms are below 1e-18
    A = 0.5 - t2 / 24.0 + t2 * t2 / 720.0;
    B = 1.0 / 6.0 - t2 / 120.0 + t2 * t2 / 5040.0;
  } else {
    const double t = sqrt(t2);
    double s, c;
    sincos(t, &s, &c);
    A = (1.0 - c) / t2;
    B = (t - s) / (t2 * t);
  }
  const double K[9] = {0, -p[2], p[1], p[2], 0, -p[0], -p[1], p[0], 0};
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const double k2 = K[i * 3] * K[j] + K[i * 3 + 1] * K[3 + j] + K[i * 3 + 2] * K[6 + j];
      J[i * 3 + j] = (i == j ? 1.0 : 0.0) + A * K[i * 3 + j] + B * k2;
    }
}

// Through the retraction: threads [0, nci) take a camera (internal order,
// BC entries), threads [nci, nci + nV3) a point coordinate.  In: lam (the
// adjoint of x_{k+1}) and delta (the step).  Out: a (the adjoint of the
// step) and lam (in place: the direct part of the adjoint of x_k).
template <int BC>
static __global__ void unroll_split_kernel(int nci, int nV3, const double* __restrict__ delta,
                                           double* __restrict__ lam, double* __restrict__ a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nci) {
    const double* dl = delta + (size_t)i * BC;
    double* l = lam + (size_t)i * BC;
    double* ai = a + (size_t)i * BC;
    double J[9], R[9];
    so3_left_jacobian(dl, J);
    so3_exp(dl, R);
    const double lw[3] = {l[0], l[1], l[2]};
#pragma unroll
    for (int r = 0; r < 3; r++) {
      ai[r] = J[r] * lw[0] + J[3 + r] * lw[1] + J[6 + r] * lw[2];
      l[r] = R[r] * lw[0] + R[3 + r] * lw[1] + R[6 + r] * lw[2];
    }
#pragma unroll
    for (int k = 3; k < BC; k++) ai[k] = l[k];
  } else if (i < nci + nV3) {
    const size_t j = (size_t)nci * BC + (i - nci);
    a[j] = lam[j];
  }
}

// d/de [w (J u) . (r + J delta)] at x (+) e along (vc, vp): the value of the
// dual part.  uc / dc (camera rows of u / delta) are null for a fixed camera,
// up / dp for a fixed point.
template <int BC>
__device__ __forceinline__ double psiphi_dir(const BaDev& d, const double* cs, const double* X, const double* vc,
                                             const double* vp, const double* uc, const double* dc,
                                             const double* up, const double* dp, double z0, double z1, double w) {
  Dual R[9], t[3], f, k1, k2, Xd[3], r[2], Jc[2 * BC], Jp[6];
  load_dual<BC>(cs, X, vc, vp, d.f_fixed, R, t, f, k1, k2, Xd);
  proj_jac_dual<BC>(R, t, f, k1, k2, Xd, z0, z1, d.cx, d.cy, r, Jc, Jp);
  Dual s = {0.0, 0.0};
#pragma unroll
  for (int i = 0; i < 2; i++) {
    Dual ju = {0.0, 0.0}, jd = {0.0, 0.0};
    if (uc) {
#pragma unroll
      for (int k = 0; k < BC; k++) {
        ju = ju + uc[k] * Jc[i * BC + k];
        jd = jd + dc[k] * Jc[i * BC + k];
      }
    }
    if (up) {
#pragma unroll
      for (int k = 0; k < 3; k++) {
        ju = ju + up[k] * Jp[i * 3 + k];
        jd = jd + dp[k] * Jp[i * 3 + k];
      }
    }
    s = s + ju * (r[i] + jd);
  }
  return w * s.d;
}

// Gradient of psi + phi w.r.t. each camera's tangent: one CTA per internal
// camera over its E-order edges, BC directions per edge.
template <int BC, int NT>
static __global__ void __launch_bounds__(NT) unroll_grad_cam_kernel(BaDev d, const double* __restrict__ uU,
                                                                    const double* __restrict__ uV,
                                                                    const double* __restrict__ dU,
                                                                    const double* __restrict__ dV,
                                                                    double* __restrict__ outU) {
  __shared__ double sh[NT / 32];
  __shared__ double cs[16];
  const int c = blockIdx.x;
  const int slot = d.cam_slot[c];
  if (threadIdx.x < 16) cs[threadIdx.x] = d.cam[(size_t)slot * 16 + threadIdx.x];
  __syncthreads();
  const double* uc = uU + (size_t)c * BC;
  const double* dc = dU + (size_t)c * BC;
  double acc[BC];
#pragma unroll
  for (int k = 0; k < BC; k++) acc[k] = 0.0;
  const int e0 = d.grp_edge_ptr[d.cam_grp_ptr[c]], e1 = d.grp_edge_ptr[d.cam_grp_ptr[c + 1]];
  for (int e = e0 + threadIdx.x; e < e1; e += NT) {
    const int ps = d.e_pt[e];
    const bool pv = ps < d.np_var;
    const double* X = d.pt + (size_t)ps * 3;
    const double z0 = d.e_obs[2 * e], z1 = d.e_obs[2 * e + 1], w = d.e_w[e];
#pragma unroll 1
    for (int k = 0; k < BC; k++) {
      double v[BC];
#pragma unroll
      for (int q = 0; q < BC; q++) v[q] = q == k ? 1.0 : 0.0;
      acc[k] += psiphi_dir<BC>(d, cs, X, v, nullptr, uc, dc, pv ? uV + (size_t)ps * 3 : nullptr,
                               pv ? dV + (size_t)ps * 3 : nullptr, z0, z1, w);
    }
  }
#pragma unroll
  for (int k = 0; k < BC; k++) {
    const double s = block_sum<NT>(acc[k], sh);
    if (threadIdx.x == 0) outU[(size_t)c * BC + k] = s;
  }
}

// Gradient of psi + phi w.r.t. each variable point: one thread per point over
// its P-order edges, 3 directions per edge.  slot2int: camera slot -> internal
// camera (-1 for a fixed camera).
template <int BC>
static __global__ void unroll_grad_pt_kernel(BaDev d, const int* __restrict__ slot2int,
                                             const double* __restrict__ uU, const double* __restrict__ uV,
                                             const double* __restrict__ dU, const double* __restrict__ dV,
                                             double* __restrict__ outV) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.np_var) return;
  double acc[3] = {0.0, 0.0, 0.0};
  const double* X = d.pt + (size_t)p * 3;
  for (int e = d.pt_edge_ptr[p]; e < d.pt_edge_ptr[p + 1]; e++) {
    const int cslot = d.p_cam[e];
    const int ci = slot2int[cslot];
    const double* cs = d.cam + (size_t)cslot * 16;
    const double z0 = d.p_obs[2 * e], z1 = d.p_obs[2 * e + 1], w = d.p_w[e];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double v[3] = {k == 0 ? 1.0 : 0.0, k == 1 ? 1.0 : 0.0, k == 2 ? 1.0 : 0.0};
      acc[k] += psiphi_dir<BC>(d, cs, X, nullptr, v, ci >= 0 ? uU + (size_t)ci * BC : nullptr,
                               ci >= 0 ? dU + (size_t)ci * BC : nullptr, uV + (size_t)p * 3,
                               dV + (size_t)p * 3, z0, z1, w);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; k++) outV[3 * (size_t)p + k] = acc[k];
}

// Per edge (E-order) at x_k, accumulated at the edge's insertion index:
//   g_obs += w J u,   g_w -= (J u) . (r + J delta).
template <int BC>
static __global__ void unroll_vjp_edge_kernel(BaDev d, const int* __restrict__ eorder,
                                              const int* __restrict__ slot2int, const double* __restrict__ uU,
                                              const double* __restrict__ uV, const double* __restrict__ dU,
                                              const double* __restrict__ dV, double* __restrict__ g_obs,
                                              double* __restrict__ g_w) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= d.ne) return;
  const int cslot = d.e_cam[e], ps = d.e_pt[e];
  const int ci = slot2int[cslot];
  double r0, r1, Jc[2 * BC], Jp[6];
  ba_project<double, BC, true, true>(d.cam + (size_t)cslot * 16, d.pt + (size_t)ps * 3, d.e_obs[2 * e],
                                     d.e_obs[2 * e + 1], d.f_fixed, d.cx, d.cy, r0, r1, Jc, Jp);
  double ju0 = 0.0, ju1 = 0.0, jd0 = 0.0, jd1 = 0.0;
  if (ci >= 0) {
    const double* u = uU + (size_t)ci * BC;
    const double* dl = dU + (size_t)ci * BC;
#pragma unroll
    for (int k = 0; k < BC; k++) {
      ju0 += Jc[k] * u[k];
      ju1 += Jc[BC + k] * u[k];
      jd0 += Jc[k] * dl[k];
      jd1 += Jc[BC + k] * dl[k];
    }
  }
  if (ps < d.np_var) {
    const double* u = uV + (size_t)ps * 3;
    const double* dl = dV + (size_t)ps * 3;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      ju0 += Jp[k] * u[k];
      ju1 += Jp[3 + k] * u[k];
      jd0 += Jp[k] * dl[k];
      jd1 += Jp[3 + k] * dl[k];
    }
  }
  const double w = d.e_w[e];
  const int q = eorder[e];
  g_obs[2 * (size_t)q] += w * ju0;
  g_obs[2 * (size_t)q + 1] += w * ju1;
  g_w[q] -= ju0 * (r0 + jd0) + ju1 * (r1 + jd1);
}

// lam -= grad
static __global__ void sub_kernel(double* __restrict__ lam, const double* __restrict__ grad, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) lam[i] -= grad[i];
}

}  // namespace nl

namespace nl {

// The adjoint of x_0 in the caller's parameters: for variable camera slot u
// (internal camera slot2int[u]) with initial state R_0 = exp(w_0),
// d/dw_0 = J_l(w_0)' lam_w (exp(w_0 + e) = exp(J_l(w_0) e) exp(w_0)); the
// other camera entries and the points are unchanged.
template <int BC>
static __global__ void unroll_to_params_kernel(int ncv, const int* __restrict__ slot2int,
                                               const double* __restrict__ cam0, const double* __restrict__ lam,
                                               double* __restrict__ g_cams) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= ncv) return;
  const double* l = lam + (size_t)slot2int[u] * BC;
  double w[3], J[9];
  so3_log_dev(cam0 + (size_t)u * 16, w);
  so3_left_jacobian(w, J);
  double* g = g_cams + (size_t)u * BC;
#pragma unroll
  for (int r = 0; r < 3; r++) g[r] = J[r] * l[0] + J[3 + r] * l[1] + J[6 + r] * l[2];
#pragma unroll
  for (int k = 3; k < BC; k++) g[k] = l[k];
}

}  // namespace nl
