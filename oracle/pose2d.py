"""FP64 CPU restatement of the SingleSection 2D scan alignment that the device
pose-graph handle (nl_pose2d_*) runs.  Test infrastructure only: the tests
compare the GPU path with it; nothing in the library imports it.

It follows:
* the point-to-line edge of nelson/tests/testGaussNewton2DScansAlign.cpp:36-120:
  e_k = (T_a m_k - T_b q_k) . (R_a n_k), cost sum e_k^2, g = (N_x, N_y,
  X_t,x N_y - X_t,y N_x), Hs = sum g g', bs = sum g e, H11 += Hs, H12 -= Hs,
  H22 += Hs, b1 += bs, b2 -= bs;
* SingleSection::computeRhoChi2Change (nelson/SingleSection.h:206-213);
* SolverCholeskyDense::computeIncrement (nelson/SolverCholeskyDense.hpp:39-67):
  diagonal * (1 + rel) + abs, factor, solve -b (a Cholesky here; the
  reference's LDLT gives the same solution for an SPD matrix);
* LevenbergMarquardt::solve (nelson/LevenbergMarquardt.hpp:36-146) and
  GaussNewton::solve (nelson/GaussNewton.hpp:32-127), step for step.
The SE(2) exponential of the left update (T <- exp(d) T) is this project's
(`problems.se2_compose`); the reference takes it from the `lie` library, which
is not available.  Parity is pinned by the reference's own test criterion on
these problems: chi2 below 1e-12 after the solve
(testGaussNewton2DScansAlign.cpp:729, `Eigen::NumTraits<double>::dummy_precision()`).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

from nelson_b200.problems import ScanAlignProblem, se2_compose

REASONS = ["SuccessAtStart", "SuccessSmallIncrement", "SuccessEpsB", "SuccessSmallResiduals",
           "SolverFailure", "MaxIterationReached", "MaxSubIterationReached"]


class Pose2DOracle:
    def __init__(self, prob: ScanAlignProblem):
        self.p = prob
        self.nv = len(prob.poses0)
        self.poses = prob.poses0.copy()
        self.bck = self.poses.copy()
        self.chi2 = 0.0
        self.H = np.zeros((3 * self.nv, 3 * self.nv))
        self.b = np.zeros(3 * self.nv)
        self.inc = np.zeros(3 * self.nv)

    def _pose(self, scan):
        return self.p.poses_true[0] if scan == 0 else self.poses[scan - 1]

    def update(self, hessian: bool):
        chi2 = 0.0
        if hessian:
            self.H[:] = 0.0
            self.b[:] = 0.0
        for i, j in self.p.edges:
            A, B = self._pose(i), self._pose(j)
            ca, sa, cb, sb = np.cos(A[2]), np.sin(A[2]), np.cos(B[2]), np.sin(B[2])
            m, n, q = self.p.scans[i], self.p.normals[i], self.p.scans[j]
            xm = np.stack([ca * m[:, 0] - sa * m[:, 1] + A[0], sa * m[:, 0] + ca * m[:, 1] + A[1]], 1)
            N = np.stack([ca * n[:, 0] - sa * n[:, 1], sa * n[:, 0] + ca * n[:, 1]], 1)
            xt = np.stack([cb * q[:, 0] - sb * q[:, 1] + B[0], sb * q[:, 0] + cb * q[:, 1] + B[1]], 1)
            err = np.sum((xm - xt) * N, 1)
            chi2 += float(err @ err)
            if hessian:
                g = np.stack([N[:, 0], N[:, 1], xt[:, 0] * N[:, 1] - xt[:, 1] * N[:, 0]], 1)
                Hs, bs = g.T @ g, g.T @ err
                ia, ib = i - 1, j - 1
                if ia >= 0:
                    self.H[3 * ia:3 * ia + 3, 3 * ia:3 * ia + 3] += Hs
                    self.b[3 * ia:3 * ia + 3] += bs
                if ib >= 0:
                    self.H[3 * ib:3 * ib + 3, 3 * ib:3 * ib + 3] += Hs
                    self.b[3 * ib:3 * ib + 3] -= bs
                if ia >= 0 and ib >= 0:
                    self.H[3 * ia:3 * ia + 3, 3 * ib:3 * ib + 3] -= Hs
                    self.H[3 * ib:3 * ib + 3, 3 * ia:3 * ia + 3] -= Hs
        self.chi2 = chi2

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

    def oplus(self):
        for u in range(self.nv):
            self.poses[u] = se2_compose(self.inc[3 * u:3 * u + 3], self.poses[u])

    def backup(self):
        self.bck = self.poses.copy()

    def rollback(self):
        self.poses = self.bck.copy()

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
