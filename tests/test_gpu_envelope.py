"""The envelope solver (nl_set_solver_kind / nl_solver_set_kind).

It factors and solves the same reduced camera system S as the dense solver
(SolverCholeskySchur, nelson/SolverCholeskySchur.hpp:136-140) but skips the
128-tiles outside S's Cholesky envelope, where the factor is zero.  With the
library's own kernels (mixed precision) every skipped operation would have
added an exact zero, so the increments and LM traces are bit-identical to the
dense solver's; the FP64 path's trailing update is cuBLAS DSYRK / DGEMM on a
smaller trailing matrix, whose internal tiling may differ, so it is held to
1e-12 instead.  Workloads: aerial grid scenes from the config-2 generator
(camera pairs near the diagonal: a narrow envelope) and a ring scene (the
ring closes, so the envelope spans the last tile rows).
"""
import dataclasses

import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import make_config

pytestmark = pytest.mark.gpu

PRECS = [N.PREC_MIXED, N.PREC_FP64]


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _same(a, b, prec):
    if prec == N.PREC_MIXED:
        return np.array_equal(a, b)
    return _rel(a, b) <= 1e-12


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("cfg,scale", [(2, 0.2), (2, 0.05), (1, 0.3)])
def test_envelope_matches_dense(prec, cfg, scale):
    p = make_config(cfg, scale)
    g = N.BAProblemGPU.from_ba(p, precision=prec)
    g.update(True)
    mu = 1e-3 * g.max_abs_hdiag()
    assert g.compute_increment(0.0, mu)
    dense = [a.copy() for a in g.increment()]
    dense_bytes = g.phase_times()["update_bytes"]
    g.set_solver_kind(N.SOLVER_ENVELOPE)
    assert g.compute_increment(0.0, mu)
    env = [a.copy() for a in g.increment()]
    env_bytes = g.phase_times()["update_bytes"]
    for a, b in zip(env, dense):
        assert _same(a, b, prec), _rel(a, b)
    if cfg == 2 and scale >= 0.2 and prec == N.PREC_MIXED:
        # grid cameras: the envelope is a few tiles wide
        assert env_bytes < 0.5 * dense_bytes, (env_bytes, dense_bytes)
    # a few LM iterations from the same start give the same trace
    traces = []
    for kind in (N.SOLVER_DENSE, N.SOLVER_ENVELOPE):
        g.set_solver_kind(kind)
        g.set_params(p.cams, p.pts)
        _, tr, _, _ = g.lm_solve(N.LMSettings(maxNumIt=4))
        traces.append(tr[:, 2].copy())
    assert _same(traces[1], traces[0], prec)
    g.close()


@pytest.mark.parametrize("prec", PRECS)
def test_envelope_solver_only_handle(oracle_lib, prec):
    p = make_config(2, 0.05)
    o = oracle_lib.Oracle.from_ba(p)
    o.update(True)
    U, V, W, bU, bV = o.hessian()
    u_rc, v_rc, w_rc = o.patterns()
    s = N.SchurSolverGPU(p.bc, p.nc_var, p.np_var, u_rc, v_rc, w_rc, precision=prec)
    s.set_hessian(U, V, W, bU, bV)
    mu = 1e-3 * o.max_abs_hdiag()
    ok, du0, dv0 = s.compute_increment(0.0, mu)
    assert ok
    s.set_solver_kind(N.SOLVER_ENVELOPE)
    ok, du1, dv1 = s.compute_increment(0.0, mu)
    assert ok
    assert _same(du1, du0, prec) and _same(dv1, dv0, prec)
    # and against the FP64 CPU oracle, with the tolerances of the parity tests
    assert o.compute_increment(0.0, mu)
    du_o, dv_o = o.increment()
    tol = 1e-10 if prec == N.PREC_FP64 else 1e-4
    assert _rel(du1, du_o) < tol and _rel(dv1, dv_o) < tol
    s.close()


def _shuffle_cameras(p, seed=5):
    """The same scene with its variable cameras in a random order."""
    q = np.random.default_rng(seed).permutation(p.nc_var)
    inv = np.argsort(q).astype(np.int32)
    return dataclasses.replace(p, cams=p.cams[q].copy(), cam_idx=inv[p.cam_idx],
                               cams_true=None if p.cams_true is None else p.cams_true[q].copy(),
                               name=p.name + "+shuffled")


@pytest.mark.parametrize("prec", PRECS)
def test_rcm_order_narrows_a_shuffled_envelope(prec):
    """nl_permute_rcm_u (the reverse Cuthill-McKee stand-in for
    permuteAMD_SchurU) puts co-observing cameras next to each other again:
    the envelope solver's trailing updates shrink, the LM trace stays the
    same up to rounding (another elimination order)."""
    p = _shuffle_cameras(make_config(2, 0.2))
    runs = {}
    for order in ("user", "rcm"):
        g = N.BAProblemGPU.from_ba(p, precision=prec, perm=None if order == "user" else "rcm")
        g.set_solver_kind(N.SOLVER_ENVELOPE)
        g.update(True)
        mu = 1e-3 * g.max_abs_hdiag()
        assert g.compute_increment(0.0, mu)
        nbytes = g.phase_times()["update_bytes"]
        perm = g.user2internal()
        g.set_params(p.cams, p.pts)
        _, tr, _, _ = g.lm_solve(N.LMSettings(maxNumIt=4))
        runs[order] = (nbytes, perm, tr[:, 2].copy())
        g.close()
    assert np.array_equal(np.sort(runs["rcm"][1]), np.arange(p.nc_var))
    assert np.array_equal(runs["user"][1], np.arange(p.nc_var))
    if prec == N.PREC_MIXED:
        assert runs["rcm"][0] < 0.5 * runs["user"][0], (runs["rcm"][0], runs["user"][0])
    c0, c1 = runs["user"][2], runs["rcm"][2]
    tol = 1e-9 if prec == N.PREC_FP64 else 1e-6
    assert len(c0) == len(c1) and np.abs(c1 - c0).max() <= tol * np.abs(c0).max()


@pytest.mark.parametrize("prec", PRECS)
def test_amd_order_gives_the_same_solve(prec):
    """nl_permute_amd_u (DoubleSection::permuteAMD_SchurU): the internal camera
    order is the host AMD order of the camera graph, and the dense and envelope
    LM traces equal the user order's up to rounding (another elimination
    order of the same S)."""
    p = _shuffle_cameras(make_config(2, 0.2))
    ref = None
    for kind in (N.SOLVER_DENSE, N.SOLVER_ENVELOPE):
        for order in ("user", "amd"):
            g = N.BAProblemGPU.from_ba(p, precision=prec, perm=None if order == "user" else "amd")
            g.set_solver_kind(kind)
            perm = g.user2internal()
            if order == "amd":
                assert np.array_equal(perm, N.amd_order_camera_graph(p.nc_var, p.np_var, p.cam_idx, p.pt_idx))
            _, tr, _, _ = g.lm_solve(N.LMSettings(maxNumIt=4))
            g.close()
            c = tr[:, 2].copy()
            if ref is None:
                ref = c
            tol = 1e-9 if prec == N.PREC_FP64 else 1e-6
            assert len(c) == len(ref) and np.abs(c - ref).max() <= tol * np.abs(ref).max(), (kind, order)


def test_rcm_order_only_before_structure():
    p = make_config(0)
    g = N.BAProblemGPU.from_ba(p, precision=N.PREC_MIXED)
    with pytest.raises(N.NelsonError):
        g._c(g.L.nl_permute_rcm_u(g.h), "nl_permute_rcm_u")
    g.close()


def test_envelope_rejects_unknown_kind():
    p = make_config(0)
    g = N.BAProblemGPU.from_ba(p, precision=N.PREC_MIXED)
    with pytest.raises(N.NelsonError):
        g.set_solver_kind(7)
    g.close()
