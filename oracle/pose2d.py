"""FP64 CPU restatement of the SingleSection 2D scan alignment that the device
pose-graph handle (nl_pose2d_*) runs.  Test infrastructure only: the tests
compare the GPU path with it; nothing in the library imports it.

It follows:
* the point-to-line edge of nelson/tests/testGaussNewton2DScansAlign.cpp:36-120:
  e_k = (T_a m_k - T_b q_k) . (R_a n_k), cost sum e_k^2, g = (N_x, N_y,
  X_t,x N_y - X_t,y N_x), Hs = sum g g', bs = sum g e, H11 += Hs, H12 -= Hs,
  H22 += Hs, b1 += bs, b2 -= bs;
* the dense increment, gain ratio and LM / GN loops of oracle/dense_lm.py.
The SE(2) exponential of the left update (T <- exp(d) T) is this project's
(`problems.se2_compose`); the reference takes it from the `lie` library, which
is not available.  Parity is pinned by the reference's own test criterion on
these problems: chi2 below 1e-12 after the solve
(testGaussNewton2DScansAlign.cpp:729, `Eigen::NumTraits<double>::dummy_precision()`).
"""
from __future__ import annotations

import numpy as np

from nelson_b200.problems import ScanAlignProblem, se2_compose
from oracle.dense_lm import REASONS, DenseLM  # noqa: F401


class Pose2DOracle(DenseLM):
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

    def oplus(self):
        for u in range(self.nv):
            self.poses[u] = se2_compose(self.inc[3 * u:3 * u + 3], self.poses[u])

    def backup(self):
        self.bck = self.poses.copy()

    def rollback(self):
        self.poses = self.bck.copy()
