import numpy as np

from nelson_b200.problems import make_config, points2d3d_fixture, project


def test_config_shapes_and_determinism():
    a = make_config(0)
    b = make_config(0)
    assert a.nc_var == 20 and a.np_var == 500 and a.bc == 6
    assert 2000 < a.ne < 3500
    assert np.array_equal(a.obs, b.obs) and np.array_equal(a.cams, b.cams)
    k = np.bincount(a.pt_idx, minlength=a.np_var)
    assert k.min() >= 3 and k.max() <= 8


def test_config2_small_scale_locality():
    p = make_config(2, 0.01)
    assert p.bc == 9
    k = np.bincount(p.pt_idx, minlength=p.np_var)
    assert k.min() >= 2 and k.max() <= 12
    gx, gy = p.meta["grid"]
    ci, cj = p.cam_idx // gy, p.cam_idx % gy
    # every observer is within 2 grid cells of the cell below the point
    x = np.clip(np.rint(p.pts_true[p.pt_idx, 0]), 0, gx - 1)
    y = np.clip(np.rint(p.pts_true[p.pt_idx, 1]), 0, gy - 1)
    assert (np.abs(ci - x) <= 2).all() and (np.abs(cj - y) <= 2).all()


def test_measurements_are_noisy_projections():
    p = make_config(0)
    z = project(p.cams_true, p.pts_true, p.cam_idx, p.pt_idx, p.bc)
    r = p.obs - z
    assert abs(r.std() - 1.0) < 0.1


def test_linear_fixture_counts():
    lp = points2d3d_fixture()
    types = [e.type for e in lp.edges]
    assert types.count(0) == 5 and types.count(1) == 3 and types.count(2) == 10 and types.count(3) == 15
