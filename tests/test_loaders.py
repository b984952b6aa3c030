"""Problem files: the reference's visibility-list format (Problem::load,
nelson/samples/Problems.cpp:8-30) and BAL-style files with observations and
parameters.  All files here are synthetic and written by the tests."""
import numpy as np
import pytest
from scipy.spatial.transform import Rotation

from nelson_b200 import problems as P


def test_pairs_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    cam = rng.integers(0, 7, size=50).astype(np.int32)
    pt = rng.integers(0, 30, size=50).astype(np.int32)
    f = tmp_path / "vis.txt"
    P.save_pairs(str(f), 7, 30, cam, pt)
    nc, npts, c2, p2 = P.load_pairs(str(f))
    assert (nc, npts) == (7, 30)
    assert np.array_equal(c2, cam) and np.array_equal(p2, pt)


def test_pairs_errors(tmp_path):
    f = tmp_path / "bad.txt"
    f.write_text("3 4 2\n0 1\n")
    with pytest.raises(ValueError):
        P.load_pairs(str(f))  # fewer pairs than announced
    f.write_text("3 4 1\n3 1\n")
    with pytest.raises(ValueError):
        P.load_pairs(str(f))  # camera index out of range
    f.write_text("")
    with pytest.raises(ValueError):
        P.load_pairs(str(f))


def test_problem_from_pairs_is_well_posed():
    rng = np.random.default_rng(1)
    cam = np.repeat(np.arange(12), 40).astype(np.int32)
    pt = rng.integers(0, 200, size=cam.size).astype(np.int32)
    p = P.problem_from_pairs(12, 200, cam, pt, bc=9, seed=3)
    assert p.ne == cam.size and p.nc_var == 12 and p.np_var == 200
    # every observed point lies in front of its camera at the true parameters
    R = P.so3_exp(p.cams_true[:, :3])
    depth = np.einsum("ej,ej->e", R[p.cam_idx, 2, :], p.pts_true[p.pt_idx]) + p.cams_true[p.cam_idx, 5]
    assert (depth > 1.0).all()
    assert np.isfinite(p.obs).all()


def _bal_cost(cams, pts, cam_idx, pt_idx, obs_bal):
    """The BAL camera model written out independently: P = R X + t,
    p = -P.xy / P.z, pixel = f (1 + k1 |p|^2 + k2 |p|^4) p."""
    R = Rotation.from_rotvec(cams[cam_idx, :3]).as_matrix()
    Pc = np.einsum("eij,ej->ei", R, pts[pt_idx]) + cams[cam_idx, 3:6]
    p = -Pc[:, :2] / Pc[:, 2:3]
    r2 = (p ** 2).sum(1, keepdims=True)
    f, k1, k2 = cams[cam_idx, 6:7], cams[cam_idx, 7:8], cams[cam_idx, 8:9]
    pred = f * (1 + k1 * r2 + k2 * r2 * r2) * p
    return float(((pred - obs_bal) ** 2).sum())


def _synthetic_bal(seed=5):
    p = P.make_config(1, 0.02)
    # a BAL file has no principal point: re-express the same scene about (0, 0)
    p.obs = p.obs - np.array([p.cx, p.cy])
    p.cx = p.cy = 0.0
    return p


def test_bal_round_trip(tmp_path):
    p = _synthetic_bal()
    f = tmp_path / "problem.bal"
    P.save_bal(str(f), p)
    q = P.load_bal(str(f))
    assert (q.nc_var, q.np_var, q.ne, q.bc, q.cx, q.cy) == (p.nc_var, p.np_var, p.ne, 9, 0.0, 0.0)
    assert np.array_equal(q.cam_idx, p.cam_idx) and np.array_equal(q.pt_idx, p.pt_idx)
    assert np.array_equal(q.obs, p.obs) and np.array_equal(q.cams, p.cams) and np.array_equal(q.pts, p.pts)


def test_bal_cost_convention(tmp_path, oracle_lib):
    """The loaded problem's cost (oracle) equals the BAL model's cost on the
    file's raw numbers."""
    p = _synthetic_bal()
    f = tmp_path / "problem.bal"
    P.save_bal(str(f), p)
    q = P.load_bal(str(f))
    raw_obs = -q.obs
    ref = _bal_cost(q.cams, q.pts, q.cam_idx, q.pt_idx, raw_obs)
    o = oracle_lib.Oracle.from_ba(q)
    assert o.update(False) == pytest.approx(ref, rel=1e-12)


def test_bal_rejects_unsupported(tmp_path):
    p = P.make_config(0)  # 6-parameter cameras, principal point (320, 240)
    with pytest.raises(ValueError):
        P.save_bal(str(tmp_path / "x.bal"), p)
    f = tmp_path / "short.bal"
    f.write_text("1 1 1\n0 0 1.0 2.0\n")
    with pytest.raises(ValueError):
        P.load_bal(str(f))
