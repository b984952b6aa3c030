"""The user-edge section's oracle (oracle/section.py) and host checks, on the CPU.

The oracle is pinned by a central-difference Jacobian of its own residuals
(H = J'J and b = J'r of the dense Hessian over all parameters), by a
Schur-complement solve of the same damped system giving the dense solve's
increment (the reduction nelson/SolverCholeskySchur.hpp:91-157 performs), and by
LM converging on the RangeScene problems for U blocks of 3, 6 and 9
parameters.  The C entry points reject bad arguments before touching a GPU.
"""
import ctypes

import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import range_scene
from oracle.section import SectionOracle, evaluate, layout


def test_layout_offsets():
    s = range_scene(6, nu=5, nv=12, obs_per_point=2, uu_edges=4)
    r_off, j_off = layout(s)
    dims = {0: (6, 3), 1: (6, 6), 2: (6, 0), 3: (3, 0)}
    for k in range(s.kind.size):
        da, db = dims[int(s.kind[k])]
        assert r_off[k + 1] - r_off[k] == s.m[k]
        assert j_off[k + 1] - j_off[k] == s.m[k] * (da + db)


@pytest.mark.parametrize("bu", [3, 6])
def test_hessian_is_jtj_of_a_finite_difference_jacobian(bu):
    s = range_scene(bu, nu=5, nv=12, obs_per_point=2, uu_edges=4, seed=7)
    o = SectionOracle(s)
    o.update(True)
    x, p = s.x0, s.p0
    r0, _ = evaluate(s, x, p)
    n = o.H.shape[0]
    nub = 5 * bu
    h = 1e-6
    Jd = np.zeros((r0.size, n))
    for c in range(n):
        dx = np.zeros(n)
        dx[c] = h
        rp = evaluate(s, x + dx[:nub].reshape(5, bu), p + dx[nub:].reshape(12, 3), False)[0]
        rm = evaluate(s, x - dx[:nub].reshape(5, bu), p - dx[nub:].reshape(12, 3), False)[0]
        Jd[:, c] = (rp - rm) / (2 * h)
    assert o.chi2 == pytest.approx(float(r0 @ r0), rel=1e-14)
    assert np.abs(Jd.T @ Jd - o.H).max() <= 1e-7 * np.abs(o.H).max()
    assert np.abs(Jd.T @ r0 - o.b).max() <= 1e-7 * np.abs(o.b).max()


def test_schur_reduction_gives_the_dense_increment():
    s = range_scene(3, nu=8, nv=40, obs_per_point=3, uu_edges=6, seed=2)
    o = SectionOracle(s)
    o.update(True)
    mu = 1e-3 * o.max_abs_hdiag()
    assert o.compute_increment(0.0, mu)
    n1 = 8 * 3
    Hd = o.H + mu * np.eye(o.H.shape[0])
    U, W, V = Hd[:n1, :n1], Hd[:n1, n1:], Hd[n1:, n1:]
    Vi = np.linalg.inv(V)
    S = U - W @ Vi @ W.T
    du = np.linalg.solve(S, -(o.b[:n1] - W @ Vi @ o.b[n1:]))
    dv = Vi @ (-o.b[n1:] - W.T @ du)
    assert np.abs(np.r_[du, dv] - o.inc).max() <= 1e-10 * np.abs(o.inc).max()


@pytest.mark.parametrize("bu", [3, 6, 9])
def test_lm_converges(bu):
    s = range_scene(bu, nu=20, nv=150, seed=bu)
    o = SectionOracle(s)
    reason, tr, it = o.lm_solve(maxNumIt=30)
    assert reason in ("SuccessSmallIncrement", "SuccessEpsB", "SuccessSmallResiduals", "MaxIterationReached")
    accepted = tr[tr[:, 7] == 1, 2]
    assert np.all(np.diff(accepted) <= 0)          # accepted steps never raise the cost
    assert accepted[-1] < 0.2 * tr[0, 2]
    assert np.abs(o.p - s.p_true).max() < 0.2


def test_entry_points_reject_bad_arguments_without_device():
    L = N.load()
    h = ctypes.c_void_p()
    assert L.nl_section_create(4, 10, 10, N.PREC_FP64, 0, ctypes.byref(h)) == 1    # bu not in 2, 3, 6, 9
    assert L.nl_section_create(3, -1, 10, N.PREC_FP64, 0, ctypes.byref(h)) == 1
    assert L.nl_section_create(3, 0, 10, N.PREC_FP64, 0, ctypes.byref(h)) == 1      # no U block
    assert L.nl_section_create(3, 10, 10, 5, 0, ctypes.byref(h)) == 1              # precision
    assert L.nl_section_destroy(None) == 1
    assert L.nl_section_update(None, 1, None) == 1
    assert L.nl_section_add_edges(None, 0, None, None, None, None) == 1
