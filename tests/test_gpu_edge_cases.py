"""Edge cases of the CUDA path against the FP64 oracle (through the C ABI).

* the solver-only drop-in (nl_solver_*) on the reference's linear 5x2D / 3x3D
  fixture (U with off-diagonal UU blocks, block size 2) and on a BA Hessian;
* per-edge weights (cost w |r|^2);
* duplicate edges (two updaters on one Hessian block, summed newest first as
  nelson/DoubleSection.hpp:349-363 orders them);
* fixed cameras and fixed points (NodeType::Fixed);
* a damping that makes the system indefinite: computeIncrement returns false
  and the increment is zero (nelson/SolverCholeskySchur.hpp:151-154);
* a problem with a single camera.
Tolerances as in test_gpu_parity: FP64 1e-12 on blocks / costs, 1e-10 on
increments; mixed 1e-6 on blocks, 1e-4 on increments.
"""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import (BAProblem, add_uniform_noise, make_config, points2d3d_fixture, ring_scene,
                                  with_fixed_nodes)

pytestmark = pytest.mark.gpu

PRECS = [N.PREC_FP64, N.PREC_MIXED]
INC_TOL = {N.PREC_FP64: 1e-10, N.PREC_MIXED: 1e-4}
H_TOL = {N.PREC_FP64: 1e-11, N.PREC_MIXED: 1e-5}


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _with_duplicates(p: BAProblem, n: int, seed=3) -> BAProblem:
    rng = np.random.default_rng(seed)
    idx = rng.choice(p.ne, size=n, replace=False)
    obs2 = p.obs[idx] + rng.normal(0, 0.3, size=(n, 2))
    return BAProblem(bc=p.bc, cams=p.cams, pts=p.pts, nc_var=p.nc_var, np_var=p.np_var,
                     cam_idx=np.concatenate([p.cam_idx, p.cam_idx[idx]]).astype(np.int32),
                     pt_idx=np.concatenate([p.pt_idx, p.pt_idx[idx]]).astype(np.int32),
                     obs=np.concatenate([p.obs, obs2]), f=p.f, cx=p.cx, cy=p.cy, name=p.name + "+dup")


def _check_problem(Orc, p, prec, lm_its=6):
    o = Orc.Oracle.from_ba(p)
    g = N.BAProblemGPU.from_ba(p, precision=prec)
    assert (o.nU, o.nV, o.nW, o.ne) == (g.nU, g.nV, g.nW, g.ne)
    for a, b in zip(o.patterns(), g.patterns()):
        assert np.array_equal(a, b)
    for a, b in zip(o.edge_uids(), g.edge_uids()):
        assert np.array_equal(a, b)
    c_o, c_g = o.update(True), g.update(True)
    assert c_g == pytest.approx(c_o, rel=1e-12)
    for a, b in zip(g.hessian(), o.hessian()):
        assert rel(a, b) < H_TOL[prec]
    mu = 1e-3 * o.max_abs_hdiag()
    assert o.compute_increment(0.0, mu) and g.compute_increment(0.0, mu)
    for a, b in zip(g.increment(), o.increment()):
        assert rel(a, b) < INC_TOL[prec]
    r_o, tr_o, _, _ = o.lm_solve(Orc.LMSettings(maxNumIt=lm_its))
    r_g, tr_g, _, _ = g.lm_solve(N.LMSettings(maxNumIt=lm_its))
    tol = 1e-9 if prec == N.PREC_FP64 else 1e-6
    assert abs(tr_g[-1, 2] - tr_o[-1, 2]) <= tol * tr_o[-1, 2]
    return o, g


@pytest.mark.parametrize("prec", PRECS)
def test_weighted_edges(oracle_lib, prec):
    p = make_config(4, 0.5)
    assert p.weight is not None
    _check_problem(oracle_lib, p, prec)[1].close()


@pytest.mark.parametrize("prec", PRECS)
def test_duplicate_edges(oracle_lib, prec):
    p = _with_duplicates(make_config(0), 200)
    _check_problem(oracle_lib, p, prec)[1].close()


@pytest.mark.parametrize("prec", PRECS)
def test_fixed_nodes(oracle_lib, prec):
    p = with_fixed_nodes(make_config(1, 0.05), 2, 40)
    o, g = _check_problem(oracle_lib, p, prec)
    cams, pts = g.get_params()
    assert np.abs(cams[p.nc_var:] - p.cams[p.nc_var:]).max() <= 1e-12
    assert np.array_equal(pts[p.np_var:], p.pts[p.np_var:])
    g.close()


def test_single_camera(oracle_lib):
    p = ring_scene(1, 60, 1, 1, 6, seed=99, name="one-cam")
    o, g = _check_problem(oracle_lib, p, N.PREC_FP64, lm_its=3)
    g.close()


@pytest.mark.parametrize("prec", PRECS)
def test_indefinite_damping_reports_failure(prec):
    p = make_config(0, 0.2)
    g = N.BAProblemGPU.from_ba(p, precision=prec)
    g.update(True)
    assert not g.compute_increment(0.0, -10.0 * g.max_abs_hdiag())
    du, dv = g.increment()
    assert not du.any() and not dv.any()
    assert g.inc_sqnorm() == 0.0
    # a sound call afterwards works again on the same handle
    assert g.compute_increment(0.0, 1e-3 * g.max_abs_hdiag())
    assert g.inc_sqnorm() > 0.0
    g.close()


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("u_diag,w_diag", [(False, False), (True, False), (False, True)])
def test_solver_only_linear_fixture(oracle_lib, prec, u_diag, w_diag):
    lp = points2d3d_fixture(u_block_diagonal=u_diag, w_block_diagonal=w_diag)
    add_uniform_noise(lp, 0.5, np.random.default_rng(5))
    o = oracle_lib.Oracle.from_linear(lp)
    o.update(True)
    U, V, W, bU, bV = o.hessian()
    u_rc, v_rc, w_rc = o.patterns()
    s = N.SchurSolverGPU(lp.bu, lp.nu_var, lp.nv_var, u_rc, v_rc, w_rc, precision=prec)
    s.set_hessian(U, V, W, bU, bV)
    assert s.max_abs_hdiag() == pytest.approx(o.max_abs_hdiag(), rel=1e-12)
    for lam in (0.0, 1e-3):
        assert o.compute_increment(0.0, lam)
        ok, du, dv = s.compute_increment(0.0, lam)
        assert ok
        du_o, dv_o = o.increment()
        assert rel(du, du_o) < INC_TOL[prec] and rel(dv, dv_o) < INC_TOL[prec]
    ok, du, dv = s.compute_increment(0.0, -1e3)
    assert not ok and not du.any() and not dv.any()
    s.close()


@pytest.mark.parametrize("prec", PRECS)
def test_solver_only_ba_hessian(oracle_lib, prec):
    p = make_config(1, 0.02)
    o = oracle_lib.Oracle.from_ba(p)
    o.update(True)
    U, V, W, bU, bV = o.hessian()
    u_rc, v_rc, w_rc = o.patterns()
    s = N.SchurSolverGPU(p.bc, p.nc_var, p.np_var, u_rc, v_rc, w_rc, precision=prec)
    s.set_hessian(U, V, W, bU, bV)
    mu = 1e-3 * o.max_abs_hdiag()
    assert o.compute_increment(0.0, mu)
    ok, du, dv = s.compute_increment(0.0, mu)
    assert ok
    du_o, dv_o = o.increment()
    assert rel(du, du_o) < INC_TOL[prec] and rel(dv, dv_o) < INC_TOL[prec]
    s.close()


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("kind", [N.SOLVER_DENSE, N.SOLVER_ENVELOPE])
def test_second_solve_on_a_reused_handle(prec, kind):
    """A handle solved once, reset with set_params and solved again gives the
    trace of a fresh handle.  The first solve's device loop leaves
    sub-iterations in flight after it finishes; whatever they leave in S must
    not reach the next solve (the FP64 path's library trailing updates run in
    them, unpredicated)."""
    p = make_config(2, 0.3)
    g = N.BAProblemGPU.from_ba(p, precision=prec)
    g.set_solver_kind(kind)
    _, tr1, it1, _ = g.lm_solve(N.LMSettings(maxNumIt=3), trace_cap=64)
    g.set_params(p.cams, p.pts)
    _, tr2, it2, _ = g.lm_solve(N.LMSettings(maxNumIt=3), trace_cap=64)
    assert it1 == it2 == 3
    assert np.array_equal(tr1[:, [0, 1, 6, 7]], tr2[:, [0, 1, 6, 7]])
    assert np.array_equal(tr1[:, 2], tr2[:, 2])     # the same kernels on the same inputs: bit-identical
    g.close()
