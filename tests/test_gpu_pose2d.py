"""The device SingleSection (nl_pose2d_*): 2D scan alignment with
point-to-line edges, against the FP64 oracle (oracle/pose2d.py).

* update(true): chi2, H and b equal the oracle's (FP64 1e-12 relative; the
  mixed handle stores H and b in FP32, 1e-6);
* LM and GN: the same termination, iteration count and per-step trace
  (chi2, mu, |delta|^2, acceptance) as the oracle while chi2 is above the
  round-off floor;
* the reference test's sections (nelson/tests/testGaussNewton2DScansAlign.cpp:
  485-730): full / sparse edges, noise / no noise, LM / pure GN / damped GN
  (relLambda 0.01), natural / AMD / shuffled internal order, dense and
  envelope solver, reach its criterion chi2 < 1e-12 after the solve;
* the mixed precision handle reaches the same criterion;
* argument and state errors.
"""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import scan_align_scene
from oracle.pose2d import Pose2DOracle

pytestmark = pytest.mark.gpu

CHI2_OK = 1e-12
NOISE = (0.01, 0.01, np.pi / 1000.0)


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
@pytest.mark.parametrize("order", ["natural", "amd", "shuffle"])
def test_update_matches_oracle(prec, order):
    p = scan_align_scene(15, 3000, noise=(0.3, 0.3, 0.1), full_edges=False, seed=9)
    perm = np.random.default_rng(2).permutation(15).astype(np.int32) if order == "shuffle" else None
    g = N.Pose2DGPU.from_scan_align(p, precision=prec, order=order, perm=perm)
    o = Pose2DOracle(p)
    o.update(True)
    chi2 = g.update(True)
    assert chi2 == pytest.approx(o.chi2, rel=1e-12)
    H, b = g.hessian()
    tol = 1e-12 if prec == N.PREC_FP64 else 1e-6
    assert np.abs(H - o.H).max() <= tol * np.abs(o.H).max()
    assert np.abs(b - o.b).max() <= tol * np.abs(o.b).max()
    assert g.update(False) == pytest.approx(o.chi2, rel=1e-12)
    assert np.array_equal(g.get_poses(), p.poses0)
    g.close()


def _trace_close(tr_g, tr_o, floor=1e-9):
    """Every row: same iteration, sub-iteration, ok and acceptance.  Rows
    whose oracle chi2 is above the floor (where the FP64 round-off of the
    residuals is far below their size): chi2, mu and |delta|^2 close."""
    assert len(tr_g) == len(tr_o)
    assert np.array_equal(tr_g[:, [0, 1, 6, 7]], tr_o[:, [0, 1, 6, 7]])
    rows = [k for k in range(len(tr_o)) if tr_o[k, 2] > floor]
    assert len(rows) >= 2
    for k in rows:
        g, o = tr_g[k], tr_o[k]
        assert g[2] == pytest.approx(o[2], rel=1e-6), (k, g, o)
        assert g[3] == pytest.approx(o[3], rel=1e-6), (k, g, o)
        assert g[5] == pytest.approx(o[5], rel=1e-5), (k, g, o)


@pytest.mark.parametrize("full", [True, False])
def test_lm_trace_parity(full):
    p = scan_align_scene(15, 3000, noise=(0.05, 0.05, 0.02), full_edges=full, seed=5)
    g = N.Pose2DGPU.from_scan_align(p)
    reason, tr, it = g.lm_solve()
    o = Pose2DOracle(p)
    r_o, tr_o, it_o = o.lm_solve()
    assert reason == r_o and it == it_o
    _trace_close(tr, tr_o)
    assert np.abs(g.get_poses() - o.poses).max() < 1e-9
    g.close()


@pytest.mark.parametrize("rel", [0.0, 0.01])
def test_gn_trace_parity(rel):
    p = scan_align_scene(15, 3000, noise=(0.05, 0.05, 0.02), full_edges=False, seed=6)
    g = N.Pose2DGPU.from_scan_align(p)
    reason, tr, it = g.gn_solve(N.GNSettings(relLambda=rel))
    o = Pose2DOracle(p)
    r_o, tr_o, it_o = o.gn_solve(relLambda=rel)
    assert reason == r_o and it == it_o
    _trace_close(tr, tr_o)
    assert np.abs(g.get_poses() - o.poses).max() < 1e-9
    g.close()


@pytest.mark.parametrize("order", ["natural", "amd", "shuffle"])
@pytest.mark.parametrize("kind", [N.SOLVER_DENSE, N.SOLVER_ENVELOPE])
def test_reference_sections(order, kind):
    for full in (True, False):
        for noise in (NOISE, (0.0, 0.0, 0.0)):
            p = scan_align_scene(15, 3000, noise=noise, full_edges=full, seed=3 + int(full))
            perm = np.random.default_rng(4).permutation(15).astype(np.int32) if order == "shuffle" else None
            for solver in ("lm", "gn", "gn_damped"):
                g = N.Pose2DGPU.from_scan_align(p, order=order, perm=perm)
                g.set_solver_kind(kind)
                if solver == "lm":
                    reason, _, _ = g.lm_solve()
                else:
                    reason, _, _ = g.gn_solve(N.GNSettings(relLambda=0.01 if solver == "gn_damped" else 0.0))
                assert reason != "SolverFailure"
                chi2 = g.update(True)
                assert chi2 < CHI2_OK, (full, noise, solver, reason, chi2)
                assert np.abs(g.get_poses() - p.poses_true[1:]).max() < 1e-6
                g.close()


def test_star_section():
    p = scan_align_scene(15, 1000, noise=NOISE, full_edges=False, seed=8)
    p.edges = [(0, i) for i in range(1, 16)]
    g = N.Pose2DGPU.from_scan_align(p)
    g.lm_solve()
    assert g.update(True) < CHI2_OK
    H, _ = g.hessian()
    for u in range(15):
        H[3 * u:3 * u + 3, 3 * u:3 * u + 3] = 0.0
    assert not H.any()
    g.close()


@pytest.mark.parametrize("kind", [N.SOLVER_DENSE, N.SOLVER_ENVELOPE])
def test_mixed_precision_reaches_the_criterion(kind):
    for full in (True, False):
        p = scan_align_scene(15, 3000, noise=NOISE, full_edges=full, seed=12)
        g = N.Pose2DGPU.from_scan_align(p, precision=N.PREC_MIXED, order="amd")
        g.set_solver_kind(kind)
        g.lm_solve()
        assert g.update(True) < CHI2_OK
        g.close()


def test_larger_pose_graph_matches_oracle():
    """400 variable poses on a chain with loop closures: U is 1,200 x 1,200
    (10 tiles of 128), factored by the tiled envelope Cholesky."""
    p = scan_align_scene(400, 60, noise=(0.02, 0.02, 0.01), full_edges=False, seed=21)
    rng = np.random.default_rng(3)
    edges = [(i, i + 1) for i in range(400)]
    for _ in range(150):
        i = int(rng.integers(0, 380))
        edges.append((i, i + int(rng.integers(2, 20))))
    p.edges = edges
    for order in ("natural", "amd", "rcm"):
        g = N.Pose2DGPU.from_scan_align(p, order=order)
        g.set_solver_kind(N.SOLVER_ENVELOPE)
        reason, tr, it = g.lm_solve()
        o = Pose2DOracle(p)
        r_o, tr_o, it_o = o.lm_solve()
        assert reason == r_o and it == it_o
        _trace_close(tr, tr_o)
        assert g.update(True) < CHI2_OK
        g.close()


def test_errors():
    p = scan_align_scene(3, 20, seed=1)
    g = N.Pose2DGPU(3, 1)
    with pytest.raises(N.NelsonError):
        g.update(True)                                       # before structure_ready
    with pytest.raises(N.NelsonError):
        g.add_edge(0, True, 0, True, p.scans[0], p.normals[0], p.scans[1])   # both fixed
    with pytest.raises(N.NelsonError):
        g.add_edge(0, False, 0, False, p.scans[0], p.normals[0], p.scans[1])  # same pose
    with pytest.raises(N.NelsonError):
        g.add_edge(3, False, 0, True, p.scans[0], p.normals[0], p.scans[1])   # out of range
    with pytest.raises(N.NelsonError):
        g.set_user2internal(np.array([0, 0, 1], np.int32))                   # not a permutation
    g.add_edge(0, True, 0, False, p.scans[0], p.normals[0], p.scans[1])
    g.structure_ready()
    with pytest.raises(N.NelsonError):
        g.add_edge(0, True, 1, False, p.scans[0], p.normals[0], p.scans[2])  # after structure_ready
    with pytest.raises(N.NelsonError):
        g.structure_ready()
    g.close()


def test_edge_without_points():
    """An edge holding no points adds nothing (its chunk record is zero)."""
    p = scan_align_scene(6, 300, noise=NOISE, full_edges=False, seed=4)
    g = N.Pose2DGPU(6, 1)
    g.set_poses(p.poses0, p.poses_true[:1])
    for i, j in p.edges:
        g.add_edge(i - 1 if i else 0, i == 0, j - 1 if j else 0, j == 0, p.scans[i], p.normals[i], p.scans[j])
    g.add_edge(0, False, 1, False, np.zeros((0, 2)), np.zeros((0, 2)), np.zeros((0, 2)))
    g.structure_ready()
    o = Pose2DOracle(p)
    o.update(True)
    assert g.update(True) == pytest.approx(o.chi2, rel=1e-12)
    H, b = g.hessian()
    assert np.abs(H - o.H).max() <= 1e-12 * np.abs(o.H).max()
    g.lm_solve()
    assert g.update(True) < CHI2_OK
    g.close()
