// host_lm.cuh -- LevenbergMarquardt / GaussNewton control on the host for the
// sections whose problem operations are host calls into device work (the
// single section of pose2d.cu, the user-edge section of section.cu).
//
// The loops restate nelson/LevenbergMarquardt.hpp:36-146 and
// nelson/GaussNewton.hpp:32-127 step for step over a problem type P with
//   update(bool hessian), chi2(), max_abs_b(), max_abs_hdiag(),
//   compute_increment(rel, abs) -> bool, inc_sqnorm(),
//   rho(mu, oldChi2) (computeRhoChi2Change with the candidate's chi2 already
//   evaluated), oplus(), backup(), rollback().
// An operation that fails throws HostError; the entry point returns its status.
// Trace records are 8 doubles (it, subit, chi2, mu, rho, |delta|^2, ok,
// accepted), as for nl_lm_solve.
#pragma once

#include <algorithm>

#include "../../include/nelson_b200.h"

namespace nl {

struct HostError {
  nl_status s;
};

inline void host_check(nl_status s) {
  if (s != NL_OK) throw HostError{s};
}

inline void trace_rec(double* trace, int cap, int* n, double it, double sub, double chi2, double mu, double rh,
                      double inc, double ok, double acc) {
  if (trace && *n < cap) {
    double* t = trace + (size_t)(*n) * 8;
    t[0] = it;
    t[1] = sub;
    t[2] = chi2;
    t[3] = mu;
    t[4] = rh;
    t[5] = inc;
    t[6] = ok;
    t[7] = acc;
  }
  (*n)++;
}

// LevenbergMarquardt::solve (nelson/LevenbergMarquardt.hpp:36-146)
template <class P>
int host_lm_loop(P& prob, const nl_lm_settings& s, double* trace, int cap, int* ntr, int* iters, int* subs,
                 double* mu_out) {
  int n = 0, iter = -1, nsub = 0;
  double mu = 0.0;
  auto finish = [&](int reason) {
    if (ntr) *ntr = std::min(n, cap);
    *iters = iter;
    *subs = nsub;
    if (mu_out) *mu_out = mu;
    return reason;
  };
  prob.update(true);
  trace_rec(trace, cap, &n, iter, 0, prob.chi2(), 0, 0, 0, 1, 1);
  if (prob.max_abs_b() <= s.epsBVector) return finish(NL_SUCCESS_AT_START);
  prob.backup();
  double oldChi2 = prob.chi2();
  mu = s.tau * prob.max_abs_hdiag();
  double curV = s.initV;
  iter = 0;
  while (iter < s.maxNumIt) {
    int subiter = 0;
    bool toRepeat = false;
    do {
      const double mu_used = mu;
      const bool ok = prob.compute_increment(0.0, mu);
      nsub++;
      const double inc = prob.inc_sqnorm();
      if (ok && iter >= s.minNumIt && inc <= s.epsIncSquare) {
        trace_rec(trace, cap, &n, iter, subiter, prob.chi2(), mu_used, 0, inc, 1, 0);
        return finish(NL_SUCCESS_SMALL_INCREMENT);
      }
      double rh = -1.0, chi2_rec = -1.0;
      if (ok) {
        prob.oplus();
        prob.update(false);
        chi2_rec = prob.chi2();
        rh = prob.rho(mu, oldChi2);
      }
      const bool acc = ok && rh > 0;
      trace_rec(trace, cap, &n, iter, subiter, chi2_rec, mu_used, rh, inc, ok ? 1 : 0, acc ? 1 : 0);
      if (acc) {
        if (iter > s.minNumIt && prob.max_abs_b() <= s.epsBVector) return finish(NL_SUCCESS_EPS_B);
        if (iter > s.minNumIt && prob.chi2() < s.epsChi2) return finish(NL_SUCCESS_SMALL_RESIDUALS);
        const double fc = 2 * rh - 1;
        double alpha = std::min(s.maxScaleFactor, 1 - fc * fc * fc);
        alpha = std::max(s.minScaleFactor, alpha);
        mu = mu * alpha;
        curV = s.initV;
      } else {
        prob.rollback();
        mu = mu * curV;
        curV = curV * s.penaltyV;
      }
      subiter++;
      if (subiter >= s.maxNumSubIt) return finish(NL_MAX_SUBITERATION_REACHED);
      toRepeat = (rh <= 0 || !ok);
    } while (toRepeat);
    prob.update(true);
    prob.backup();
    oldChi2 = prob.chi2();
    iter++;
  }
  return finish(NL_MAX_ITERATION_REACHED);
}

// GaussNewton::solve (nelson/GaussNewton.hpp:32-127)
template <class P>
int host_gn_loop(P& prob, const nl_gn_settings& s, double* trace, int cap, int* ntr, int* iters) {
  int n = 0, iter = -1;
  auto finish = [&](int reason) {
    if (ntr) *ntr = std::min(n, cap);
    *iters = iter;
    return reason;
  };
  prob.update(true);
  trace_rec(trace, cap, &n, iter, 0, prob.chi2(), 0, 0, 0, 1, 1);
  if (prob.max_abs_b() <= s.epsBVector) return finish(NL_SUCCESS_AT_START);
  iter = 0;
  while (iter < s.maxNumIt) {
    const bool ok = prob.compute_increment(s.relLambda, s.absLambda);
    const double inc = prob.inc_sqnorm();
    if (!ok) {
      trace_rec(trace, cap, &n, iter, 0, -1, 0, 0, inc, 0, 0);
      return finish(NL_SOLVER_FAILURE);
    }
    if (iter >= s.minNumIt && inc <= s.epsIncSquare) {
      trace_rec(trace, cap, &n, iter, 0, prob.chi2(), 0, 0, inc, 1, 0);
      return finish(NL_SUCCESS_SMALL_INCREMENT);
    }
    prob.oplus();
    prob.update(true);
    trace_rec(trace, cap, &n, iter, 0, prob.chi2(), 0, 0, inc, 1, 1);
    if (iter > s.minNumIt && prob.max_abs_b() <= s.epsBVector) return finish(NL_SUCCESS_EPS_B);
    if (iter > s.minNumIt && prob.chi2() < s.epsChi2) return finish(NL_SUCCESS_SMALL_RESIDUALS);
    iter++;
  }
  return finish(NL_MAX_ITERATION_REACHED);
}

}  // namespace nl
