"""Dense FP64 increment and LevenbergMarquardt / GaussNewton loops shared by
the CPU oracles of the single section (oracle/pose2d.py) and of the
user-edge section (oracle/section.py).  Test infrastructure only.

A subclass provides update(hessian) (setting self.chi2 and, with hessian,
the dense self.H and self.b over all its parameters), oplus() (applying
self.inc), backup() and rollback().  This module follows:
* computeRhoChi2Change (nelson/SingleSection.h:206-213,
  nelson/DoubleSection.h:300-311): (old - new) / delta' (mu delta - b);
* SolverCholeskyDense::computeIncrement (nelson/SolverCholeskyDense.hpp:39-67):
  diagonal * (1 + rel) + abs, factor, solve -b (a Cholesky here; the
  reference's LDLT gives the same solution for an SPD matrix, and on the
  damped Hessian [U W; W' V] the Schur complement solve of
  nelson/SolverCholeskySchur.hpp:91-157 gives it too, damping both
  diagonals);
* LevenbergMarquardt::solve (nelson/LevenbergMarquardt.hpp:36-146) and
  GaussNewton::solve (nelson/GaussNewton.hpp:32-127), step for step.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

REASONS = ["SuccessAtStart", "SuccessSmallIncrement", "SuccessEpsB", "SuccessSmallResiduals",
           "SolverFailure", "MaxIterationReached", "MaxSubIterationReached"]


class DenseLM:
    def max_abs_b(self):
        return float(np.abs(self.b).max()) if self.b.size else 0.0

    def max_abs_hdiag(self):
        return float(np.abs(np.diag(self.H)).max()) if self.H.size else 0.0

    def compute_increment(self, rel, abs_):
        Hd = self.H.copy()
        d = np.diag(Hd) * (1.0 + rel) + abs_
        np.fill_diagonal(Hd, d)
        try:
            c = sla.cho_factor(Hd, lower=True, check_finite=False)
        except np.linalg.LinAlgError:
            self.inc[:] = 0.0
            return False
        self.inc = sla.cho_solve(c, -self.b, check_finite=False)
        return True

    def inc_sqnorm(self):
        return float(self.inc @ self.inc)

    def rho(self, mu, old_chi2):
        return (old_chi2 - self.chi2) / float(self.inc @ (mu * self.inc - self.b))

    # LevenbergMarquardt::solve (nelson/LevenbergMarquardt.hpp:36-146); defaults of
    # nelson/LevenbergMarquardt.cpp:6-19
    def lm_solve(self, maxNumIt=100, maxNumSubIt=10, minNumIt=0, epsBVector=1e-15, epsIncSquare=1e-30,
                 epsChi2=1e-15, tau=1e-3, penaltyV=2.0, initV=2.0, maxScaleFactor=2.0 / 3.0,
                 minScaleFactor=1.0 / 3.0):
        tr = []
        it = -1
        self.update(True)
        tr.append((it, 0, self.chi2, 0, 0, 0, 1, 1))
        if self.max_abs_b() <= epsBVector:
            return "SuccessAtStart", np.array(tr), it
        self.backup()
        old = self.chi2
        mu = tau * self.max_abs_hdiag()
        cur_v = initV
        it = 0
        while it < maxNumIt:
            sub = 0
            while True:
                mu_used = mu
                ok = self.compute_increment(0.0, mu)
                inc = self.inc_sqnorm()
                if ok and it >= minNumIt and inc <= epsIncSquare:
                    tr.append((it, sub, self.chi2, mu_used, 0, inc, 1, 0))
                    return "SuccessSmallIncrement", np.array(tr), it
                rh, chi2_rec = -1.0, -1.0
                if ok:
                    self.oplus()
                    self.update(False)
                    chi2_rec = self.chi2
                    rh = self.rho(mu, old)
                acc = ok and rh > 0
                tr.append((it, sub, chi2_rec, mu_used, rh, inc, int(ok), int(acc)))
                if acc:
                    if it > minNumIt and self.max_abs_b() <= epsBVector:
                        return "SuccessEpsB", np.array(tr), it
                    if it > minNumIt and self.chi2 < epsChi2:
                        return "SuccessSmallResiduals", np.array(tr), it
                    fc = 2 * rh - 1
                    alpha = max(minScaleFactor, min(maxScaleFactor, 1 - fc ** 3))
                    mu *= alpha
                    cur_v = initV
                else:
                    self.rollback()
                    mu *= cur_v
                    cur_v *= penaltyV
                sub += 1
                if sub >= maxNumSubIt:
                    return "MaxSubIterationReached", np.array(tr), it
                if not (rh <= 0 or not ok):
                    break
            self.update(True)
            self.backup()
            old = self.chi2
            it += 1
        return "MaxIterationReached", np.array(tr), it

    # GaussNewton::solve (nelson/GaussNewton.hpp:32-127); defaults of nelson/GaussNewton.cpp:12-22
    def gn_solve(self, maxNumIt=100, minNumIt=0, epsBVector=1e-15, epsIncSquare=1e-30, epsChi2=1e-15,
                 absLambda=0.0, relLambda=0.0):
        tr = []
        it = -1
        self.update(True)
        tr.append((it, 0, self.chi2, 0, 0, 0, 1, 1))
        if self.max_abs_b() <= epsBVector:
            return "SuccessAtStart", np.array(tr), it
        it = 0
        while it < maxNumIt:
            ok = self.compute_increment(relLambda, absLambda)
            inc = self.inc_sqnorm()
            if not ok:
                tr.append((it, 0, -1, 0, 0, inc, 0, 0))
                return "SolverFailure", np.array(tr), it
            if it >= minNumIt and inc <= epsIncSquare:
                tr.append((it, 0, self.chi2, 0, 0, inc, 1, 0))
                return "SuccessSmallIncrement", np.array(tr), it
            self.oplus()
            self.update(True)
            tr.append((it, 0, self.chi2, 0, 0, inc, 1, 1))
            if it > minNumIt and self.max_abs_b() <= epsBVector:
                return "SuccessEpsB", np.array(tr), it
            if it > minNumIt and self.chi2 < epsChi2:
                return "SuccessSmallResiduals", np.array(tr), it
            it += 1
        return "MaxIterationReached", np.array(tr), it
