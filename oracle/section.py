"""FP64 CPU oracle of the user-edge section (nl_section_*) on the RangeScene
problem of nelson_b200.problems.  Test infrastructure only.

`evaluate` computes every edge's residual and Jacobian blocks in the
section's layout (edge e's residual at r_off[e], its J_a (m x dim_a,
row-major) at j_off[e], then J_b), so the GPU tests can also hand these very
arrays to the section.  The oracle itself accumulates the dense Hessian over
all parameters [x (user order) ; p] -- the Hessian that BaseSection::
updateHessianBlocks (nelson/BaseSection.cpp:5-86) assembles block by block --
and runs the dense LM / GN of oracle/dense_lm.py on it.
"""
from __future__ import annotations

import numpy as np

from nelson_b200.problems import RangeScene
from oracle.dense_lm import REASONS, DenseLM  # noqa: F401


def layout(s: RangeScene):
    """Per-edge offsets (ne + 1) into r and J."""
    dims_a = np.where(s.kind == 3, 3, s.bu)
    dims_b = np.where(s.kind == 0, 3, np.where(s.kind == 1, s.bu, 0))
    r_off = np.concatenate([[0], np.cumsum(s.m)]).astype(np.int64)
    j_off = np.concatenate([[0], np.cumsum(s.m * (dims_a + dims_b))]).astype(np.int64)
    return r_off, j_off


def evaluate(s: RangeScene, x, p, jacobians=True):
    """(r, J) of every edge at (x, p), in the section's layout."""
    r_off, j_off = layout(s)
    r = np.zeros(r_off[-1])
    J = np.zeros(j_off[-1])
    bu = s.bu
    for k in range(s.kind.size):
        ro, jo = r_off[k], j_off[k]
        if s.kind[k] == 0:
            u, v = s.a[k], s.b[k]
            diff = x[u, :3] - p[v]
            rng = np.linalg.norm(diff)
            r[ro] = rng - s.d[k]
            r[ro + 1] = s.avec[k] @ diff + s.cvec[k] @ x[u, 3:] - s.e[k]
            if jacobians:
                Ja = np.zeros((2, bu))
                Ja[0, :3] = diff / rng
                Ja[1, :3] = s.avec[k]
                Ja[1, 3:] = s.cvec[k]
                Jb = np.stack([-diff / rng, -s.avec[k]])
                J[jo:jo + 2 * bu] = Ja.ravel()
                J[jo + 2 * bu:jo + 2 * bu + 6] = Jb.ravel()
        elif s.kind[k] == 1:
            i, j = s.a[k], s.b[k]
            r[ro:ro + bu] = x[i] - x[j] - s.delta[k]
            if jacobians:
                J[jo:jo + bu * bu] = np.eye(bu).ravel()
                J[jo + bu * bu:jo + 2 * bu * bu] = -np.eye(bu).ravel()
        elif s.kind[k] == 2:
            u = s.a[k]
            r[ro:ro + bu] = s.w[k] * (x[u] - s.prior[k])
            if jacobians:
                J[jo:jo + bu * bu] = (s.w[k] * np.eye(bu)).ravel()
        else:
            v = s.a[k]
            r[ro:ro + 3] = s.w[k] * (p[v] - s.prior[k, :3])
            if jacobians:
                J[jo:jo + 9] = (s.w[k] * np.eye(3)).ravel()
    return r, J


class SectionOracle(DenseLM):
    def __init__(self, s: RangeScene):
        self.s = s
        self.x = s.x0.copy()
        self.p = s.p0.copy()
        self.nu, self.nv, self.bu = len(s.x0), len(s.p0), s.bu
        n = self.nu * self.bu + 3 * self.nv
        self.H = np.zeros((n, n))
        self.b = np.zeros(n)
        self.inc = np.zeros(n)
        self.chi2 = 0.0
        self.r_off, self.j_off = layout(s)

    def _cols(self, k, side):
        kind, bu, nub = self.s.kind[k], self.bu, self.nu * self.bu
        if kind == 3 or (kind == 0 and side == 1):
            v = self.s.a[k] if kind == 3 else self.s.b[k]
            return np.arange(nub + 3 * v, nub + 3 * v + 3)
        u = self.s.a[k] if side == 0 else self.s.b[k]
        return np.arange(bu * u, bu * u + bu)

    def update(self, hessian: bool):
        r, J = evaluate(self.s, self.x, self.p, hessian)
        self.chi2 = float(r @ r)
        if not hessian:
            return
        self.H[:] = 0.0
        self.b[:] = 0.0
        for k in range(self.s.kind.size):
            m = int(self.s.m[k])
            ro, jo = self.r_off[k], self.j_off[k]
            ca = self._cols(k, 0)
            blocks = [(ca, J[jo:jo + m * ca.size].reshape(m, ca.size))]
            if self.s.kind[k] in (0, 1):
                cb = self._cols(k, 1)
                o = jo + m * ca.size
                blocks.append((cb, J[o:o + m * cb.size].reshape(m, cb.size)))
            rk = r[ro:ro + m]
            for ci, Ji in blocks:
                self.b[ci] += Ji.T @ rk
                for cj, Jj in blocks:
                    self.H[np.ix_(ci, cj)] += Ji.T @ Jj

    def oplus(self):
        nub = self.nu * self.bu
        self.x = self.x + self.inc[:nub].reshape(self.nu, self.bu)
        self.p = self.p + self.inc[nub:].reshape(self.nv, 3)

    def backup(self):
        self.bck = (self.x.copy(), self.p.copy())

    def rollback(self):
        self.x, self.p = self.bck[0].copy(), self.bck[1].copy()
