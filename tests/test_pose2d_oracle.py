"""The 2D scan alignment oracle (oracle/pose2d.py) on the CPU.

Pinned two ways:
* its Hessian and gradient equal J'J and J'e of a finite-difference Jacobian
  of the point-to-line residuals under the left SE(2) perturbation
  (the edge of nelson/tests/testGaussNewton2DScansAlign.cpp:36-120);
* on the reference test's problem (15 variable poses, one fixed, 3,000
  points per scan, noise sigma (0.01, 0.01, pi / 1000) or none, full or
  sparse edges, testGaussNewton2DScansAlign.cpp:485-730) LM, pure GN and
  damped GN (relLambda 0.01) reach the test's criterion, chi2 below 1e-12
  after the solve (testGaussNewton2DScansAlign.cpp:728).
Plus the host-side argument checks of the device handle (no GPU needed).
"""
import ctypes

import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import scan_align_scene, se2_compose
from oracle.pose2d import Pose2DOracle

CHI2_OK = 1e-12   # Eigen::NumTraits<double>::dummy_precision()


def _residuals(prob, poses):
    out = []
    for i, j in prob.edges:
        A = prob.poses_true[0] if i == 0 else poses[i - 1]
        B = prob.poses_true[0] if j == 0 else poses[j - 1]
        ca, sa, cb, sb = np.cos(A[2]), np.sin(A[2]), np.cos(B[2]), np.sin(B[2])
        m, n, q = prob.scans[i], prob.normals[i], prob.scans[j]
        xm = np.stack([ca * m[:, 0] - sa * m[:, 1] + A[0], sa * m[:, 0] + ca * m[:, 1] + A[1]], 1)
        nn = np.stack([ca * n[:, 0] - sa * n[:, 1], sa * n[:, 0] + ca * n[:, 1]], 1)
        xt = np.stack([cb * q[:, 0] - sb * q[:, 1] + B[0], sb * q[:, 0] + cb * q[:, 1] + B[1]], 1)
        out.append(np.sum((xm - xt) * nn, 1))
    return np.concatenate(out)


def test_hessian_is_jtj_of_the_left_perturbation():
    p = scan_align_scene(4, 40, noise=(0.3, 0.3, 0.2), full_edges=True, seed=11)
    o = Pose2DOracle(p)
    o.update(True)
    e0 = _residuals(p, o.poses)
    assert o.chi2 == pytest.approx(float(e0 @ e0), rel=1e-13)
    nv = len(p.poses0)
    J = np.zeros((e0.size, 3 * nv))
    h = 1e-6
    for u in range(nv):
        for k in range(3):
            d = np.zeros(3)
            d[k] = h
            pp, pm = o.poses.copy(), o.poses.copy()
            pp[u] = se2_compose(d, o.poses[u])
            pm[u] = se2_compose(-d, o.poses[u])
            J[:, 3 * u + k] = (_residuals(p, pp) - _residuals(p, pm)) / (2 * h)
    H, b = J.T @ J, J.T @ e0
    assert np.abs(o.H - H).max() <= 1e-6 * np.abs(H).max()
    assert np.abs(o.b - b).max() <= 1e-6 * np.abs(b).max()


@pytest.mark.parametrize("full", [True, False])
@pytest.mark.parametrize("noise", [(0.01, 0.01, np.pi / 1000.0), (0.0, 0.0, 0.0)])
def test_reference_sections_converge(full, noise):
    p = scan_align_scene(15, 3000, noise=noise, full_edges=full, seed=5)
    for solve in (lambda o: o.lm_solve(), lambda o: o.gn_solve(), lambda o: o.gn_solve(relLambda=0.01)):
        o = Pose2DOracle(p)
        reason, tr, _ = solve(o)
        assert reason in ("SuccessSmallIncrement", "SuccessSmallResiduals", "SuccessEpsB", "SuccessAtStart")
        o.update(True)
        assert o.chi2 < CHI2_OK
        assert np.abs(o.poses - p.poses_true[1:]).max() < 1e-6


def test_star_section_converges():
    """Only the edges to the fixed pose (the block-diagonal Hessian of the
    reference's BlockDiagonal section types)."""
    p = scan_align_scene(15, 500, full_edges=False, seed=7)
    p.edges = [(0, i) for i in range(1, 16)]
    o = Pose2DOracle(p)
    o.lm_solve()
    o.update(True)
    assert o.chi2 < CHI2_OK
    off = o.H.copy()
    for u in range(15):
        off[3 * u:3 * u + 3, 3 * u:3 * u + 3] = 0.0
    assert not off.any()


def test_handle_argument_checks_without_device():
    L = N.load()
    h = ctypes.c_void_p()
    assert L.nl_pose2d_create(-1, 1, N.PREC_FP64, 0, ctypes.byref(h)) == 1      # NL_ERR_ARG
    assert L.nl_pose2d_create(0, 1, N.PREC_FP64, 0, ctypes.byref(h)) == 1       # no variable pose
    assert L.nl_pose2d_create(3, 1, 7, 0, ctypes.byref(h)) == 1                 # unknown precision
    assert L.nl_pose2d_create(3, 1, N.PREC_FP64, 0, None) == 1
    assert L.nl_pose2d_destroy(None) == 1
    assert L.nl_pose2d_update(None, 1, None) == 1
