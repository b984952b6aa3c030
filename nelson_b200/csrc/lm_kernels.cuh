// lm_kernels.cuh -- LevenbergMarquardt / GaussNewton control kept on the device.
//
// The state machine of LevenbergMarquardt::solve
// (nelson/LevenbergMarquardt.hpp:36-146) split into single-thread kernels
// that read and write an LmDev record in device memory, so one sub-iteration
// is a fixed launch sequence (capturable in a CUDA graph) whose kernels test
// flags instead of the host branching:
//   lm_begin_kernel    active = !done; clears the solver status word
//   [computeIncrement kernels, predicated on `active`]
//   lm_inc_kernel      |inc|^2, den = inc'(mu inc - b); SuccessSmallIncrement test;
//                      `apply` = active && solve ok && !done
//   [oplus + cost kernels, predicated on `apply`]
//   lm_decide_kernel   rho, accept / reject, mu / v update, termination tests;
//                      `rollback` and `do_jac` flags
//   [rollback copies on `rollback`; Jacobian pass on `do_jac`]
//   lm_after_jac_kernel oldChi2 = chi2, iter++, MaxIterationReached test
#pragma once

#include "nl_common.cuh"

namespace nl {

struct LmDev {
  // settings (LevenbergMarquardtSettings / GaussNewtonSettings)
  int maxNumIt, maxNumSubIt, minNumIt, gn;
  double epsBVector, epsIncSquare, epsChi2, tau, penaltyV, initV, maxScale, minScale;
  double gnRel, gnAbs;
  // state
  double mu, curV, oldChi2, chi2, chi2_new, rho, incSq, den, maxAbsB, maxAbsHDiag;
  double lam[2];  // (relLambda, absLambda) read by the solver kernels
  int iter, subiter, nsub, done, reason, solve_ok;
  int active, apply, rollback, do_jac, accepted;
  int trace_n, trace_cap;
  int status;     // solver status bits of the current sub-iteration
};

static __global__ void lm_begin_kernel(LmDev* s) {
  s->active = s->done ? 0 : 1;
  s->status = 0;
  s->apply = 0;
  s->rollback = 0;
  s->do_jac = 0;
  if (!s->done) {
    if (s->gn) {
      s->lam[0] = s->gnRel;
      s->lam[1] = s->gnAbs;
    } else {
      s->lam[0] = 0.0;
      s->lam[1] = s->mu;
    }
  }
}

__device__ inline void lm_trace(LmDev* s, double* trace, double it, double sub, double chi2, double mu, double rho,
                                double inc, double ok, double acc) {
  if (trace && s->trace_n < s->trace_cap) {
    double* t = trace + (size_t)s->trace_n * NL_TRACE_STRIDE;
    t[0] = it; t[1] = sub; t[2] = chi2; t[3] = mu; t[4] = rho; t[5] = inc; t[6] = ok; t[7] = acc;
  }
  s->trace_n++;
}

// Partial sums of |inc|^2 and inc'(mu inc - b) over CTAs.
template <typename T, int NT>
static __global__ void __launch_bounds__(NT) inc_dot_kernel(const double* __restrict__ incU, const T* __restrict__ bU,
                                                     int nu, const double* __restrict__ incV,
                                                     const T* __restrict__ bV, int nv, const LmDev* __restrict__ s,
                                                     double* __restrict__ part) {
  __shared__ double sh[NT / 32];
  if (!s->active) return;
  const double mu = s->gn ? 0.0 : s->mu;
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * NT + threadIdx.x; i < nu + nv; i += gridDim.x * NT) {
    double x, g;
    if (i < nu) {
      x = incU[i];
      g = (double)bU[i];
    } else {
      x = incV[i - nu];
      g = (double)bV[i - nu];
    }
    a += x * x;
    b += x * (mu * x - g);
  }
  a = block_sum<NT>(a, sh);
  b = block_sum<NT>(b, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

static __global__ void lm_inc_kernel(LmDev* s, const double* __restrict__ part, int nparts, double* trace) {
  if (!s->active) return;
  double a = 0.0, b = 0.0;
  for (int i = 0; i < nparts; i++) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  s->solve_ok = (s->status & (ST_VINV_FAIL | ST_CHOL_FAIL | ST_SPIN_TIMEOUT)) == 0;
  if (!isfinite(a)) s->solve_ok = 0;
  s->incSq = s->solve_ok ? a : 0.0;
  s->den = b;
  if (s->gn) {
    // GaussNewton::solve (nelson/GaussNewton.hpp:64-87)
    if (!s->solve_ok) {
      lm_trace(s, trace, s->iter, 0, -1, 0, 0, s->incSq, 0, 0);
      s->done = 1;
      s->reason = NL_SOLVER_FAILURE;
      return;
    }
    if (s->iter >= s->minNumIt && s->incSq <= s->epsIncSquare) {
      lm_trace(s, trace, s->iter, 0, s->chi2, 0, 0, s->incSq, 1, 0);
      s->done = 1;
      s->reason = NL_SUCCESS_SMALL_INCREMENT;
      return;
    }
    s->apply = 1;
    return;
  }
  // LevenbergMarquardt.hpp:73-75
  if (s->solve_ok && s->iter >= s->minNumIt && s->incSq <= s->epsIncSquare) {
    lm_trace(s, trace, s->iter, s->subiter, s->chi2, s->mu, 0, s->incSq, 1, 0);
    s->done = 1;
    s->reason = NL_SUCCESS_SMALL_INCREMENT;
    return;
  }
  s->apply = s->solve_ok;
}

// LevenbergMarquardt.hpp:78-129 (LM) / GaussNewton.hpp:89-123 (GN).
static __global__ void lm_decide_kernel(LmDev* s, double* trace) {
  if (!s->active || s->done) return;
  if (s->gn) {
    // oplus + update(true) already ran: chi2_new and maxAbsB are current
    s->nsub++;
    s->do_jac = 1;  // the Jacobian pass runs on the accepted state
    return;
  }
  double rho = -1.0;
  if (s->apply) rho = (s->oldChi2 - s->chi2_new) / s->den;
  s->rho = rho;
  const bool acc = s->apply && rho > 0.0;
  s->accepted = acc ? 1 : 0;
  lm_trace(s, trace, s->iter, s->subiter, s->apply ? s->chi2_new : -1.0, s->mu, rho, s->incSq, s->solve_ok, acc);
  s->nsub++;
  if (acc) {
    s->chi2 = s->chi2_new;
    if (s->iter > s->minNumIt && s->maxAbsB <= s->epsBVector) {
      s->done = 1;
      s->reason = NL_SUCCESS_EPS_B;
      return;
    }
    if (s->iter > s->minNumIt && s->chi2_new < s->epsChi2) {
      s->done = 1;
      s->reason = NL_SUCCESS_SMALL_RESIDUALS;
      return;
    }
    const double fc = 2.0 * rho - 1.0;
    double alpha = fmin(s->maxScale, 1.0 - fc * fc * fc);
    alpha = fmax(s->minScale, alpha);
    s->mu = s->mu * alpha;
    s->curV = s->initV;
  } else {
    s->rollback = 1;
    s->mu = s->mu * s->curV;
    s->curV = s->curV * s->penaltyV;
  }
  s->subiter++;
  if (s->subiter >= s->maxNumSubIt) {
    s->done = 1;
    s->reason = NL_MAX_SUBITERATION_REACHED;
    return;
  }
  if (acc) s->do_jac = 1;
}

static __global__ void lm_after_jac_kernel(LmDev* s, const double* __restrict__ chi2, double* trace) {
  if (!s->do_jac) return;
  s->chi2 = *chi2;
  s->oldChi2 = s->chi2;
  if (s->gn) {
    // GaussNewton.hpp:104-123
    lm_trace(s, trace, s->iter, 0, s->chi2, 0, 0, s->incSq, 1, 1);
    if (s->iter > s->minNumIt && s->maxAbsB <= s->epsBVector) {
      s->done = 1;
      s->reason = NL_SUCCESS_EPS_B;
      return;
    }
    if (s->iter > s->minNumIt && s->chi2 < s->epsChi2) {
      s->done = 1;
      s->reason = NL_SUCCESS_SMALL_RESIDUALS;
      return;
    }
  }
  s->iter++;
  s->subiter = 0;
  if (s->iter >= s->maxNumIt) {
    s->done = 1;
    s->reason = NL_MAX_ITERATION_REACHED;
  }
}

// max |x| over two arrays (CTA partials).
template <typename T, int NT>
static __global__ void __launch_bounds__(NT) maxabs_kernel(const T* __restrict__ a, int na, const T* __restrict__ b, int nb,
                                                    double* __restrict__ part, const int* __restrict__ active) {
  __shared__ double sh[NT / 32];
  if (active && !*active) return;
  double m = 0.0;
  for (int i = blockIdx.x * NT + threadIdx.x; i < na + nb; i += gridDim.x * NT) {
    const double v = fabs((double)(i < na ? a[i] : b[i - na]));
    m = fmax(m, v);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int i = 0; i < NT / 32; i++) r = fmax(r, sh[i]);
    part[blockIdx.x] = r;
  }
}

static __global__ void max_finalize_kernel(const double* __restrict__ part, int n, double* __restrict__ out,
                                    const int* __restrict__ active) {
  if (active && !*active) return;
  double m = 0.0;
  for (int i = 0; i < n; i++) m = fmax(m, part[i]);
  *out = m;
}

// max |diag| over the U diagonal blocks and the V blocks (SolverCholeskySchur::maxAbsHDiag).
template <typename T, int BC>
static __global__ void hdiag_kernel(const T* __restrict__ U, const int* __restrict__ u_diag_uid, int nci,
                             const T* __restrict__ V, const int* __restrict__ v_uid, int np,
                             double* __restrict__ part) {
  __shared__ double sh[8];
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nci + np; i += gridDim.x * blockDim.x) {
    if (i < nci) {
      const int q = u_diag_uid[i];
      if (q >= 0)
        for (int r = 0; r < BC; r++) m = fmax(m, fabs((double)U[(size_t)q * Layout<T, BC>::U + r * BC + r]));
    } else {
      const int q = v_uid[i - nci];
      if (q >= 0)
        for (int r = 0; r < 3; r++) m = fmax(m, fabs((double)V[(size_t)q * Layout<T, BC>::V + r * 3 + r]));
    }
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) r = fmax(r, sh[i]);
    part[blockIdx.x] = r;
  }
}

static __global__ void zero_if_failed_kernel(double* __restrict__ x, int n, const int* __restrict__ status,
                                      const int* __restrict__ active) {
  if (active && !*active) return;
  if ((*status & (ST_VINV_FAIL | ST_CHOL_FAIL | ST_SPIN_TIMEOUT)) == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = 0.0;
}

// copy predicated on a device flag (backup / rollback of parameters)
static __global__ void copy_if_kernel(double* __restrict__ dst, const double* __restrict__ src, size_t n,
                               const int* __restrict__ flag) {
  if (flag && !*flag) return;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

}  // namespace nl
