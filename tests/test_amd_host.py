"""The approximate minimum degree order (nl_amd_order, nl_amd_order_camera_graph,
the host functions behind nl_permute_amd_u) and the symbolic fill count
(nl_symbolic_fill), on the CPU.

The reference orders with Eigen::AMDOrdering (DoubleSection::permuteAMD_SchurU,
nelson/DoubleSection.hpp:30-63; SingleSection::permuteAMD,
nelson/SingleSection.hpp:33-52).  Eigen is not available here, so the order is
pinned by what any minimum degree order must do and by the fill it gives:
* always a permutation (empty, isolated, duplicate and two-triangle input);
* no fill on graphs that have a perfect elimination order (trees, a star
  whose hub is a dense row, a clique);
* on a 2D grid, the fill of an exact (non-approximate) minimum degree order
  within 10%, and well below the natural and reverse Cuthill-McKee fills;
* on bundle adjustment camera graphs (about 50 neighbours per camera) the
  fill of an exact minimum degree order within 5% and below the natural
  order's (reverse Cuthill-McKee, printed beside it, is as good or a little
  better on these band-like graphs: 5,070 against 5,548 on the 144-camera
  grid scene).
The fill count itself is checked against an explicit symbolic elimination.
"""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import grid_scene, make_config


def _adj(n, r, c):
    a = [set() for _ in range(n)]
    for i, j in zip(r, c):
        if i != j:
            a[i].add(j)
            a[j].add(i)
    return a


def _fill_by_elimination(n, r, c, perm):
    """Entries below the diagonal of the factor, by eliminating in order."""
    a = _adj(n, r, c)
    order = np.argsort(perm)
    pos = np.asarray(perm)
    total = 0
    for v in order:
        higher = {u for u in a[v] if pos[u] > pos[v]}
        total += len(higher)
        for u in higher:
            a[u] |= higher - {u}
    return total


def _exact_min_degree(n, r, c):
    a = _adj(n, r, c)
    alive = set(range(n))
    perm = np.empty(n, np.int32)
    for k in range(n):
        v = min(alive, key=lambda x: (len(a[x]), x))
        nb = a[v]
        for u in nb:
            a[u] |= nb - {u}
            a[u].discard(v)
        alive.discard(v)
        perm[v] = k
    return perm


def _grid(k):
    idx = np.arange(k * k).reshape(k, k)
    r = np.concatenate([idx[:, :-1].ravel(), idx[:-1, :].ravel()])
    c = np.concatenate([idx[:, 1:].ravel(), idx[1:, :].ravel()])
    return k * k, r, c


def _camera_graph(nc, cam, pt):
    order = np.argsort(pt, kind="stable")
    cam, pt = cam[order], pt[order]
    starts = np.flatnonzero(np.r_[True, pt[1:] != pt[:-1]])
    ends = np.r_[starts[1:], pt.size]
    pairs = set()
    for a, b in zip(starts, ends):
        u = np.unique(cam[a:b])
        for i in range(u.size):
            for j in range(i + 1, u.size):
                pairs.add((int(u[i]), int(u[j])))
    p = np.array(sorted(pairs), np.int32).reshape(-1, 2)
    return p[:, 0], p[:, 1]


def _is_perm(p, n):
    return np.array_equal(np.sort(p), np.arange(n))


def test_symbolic_fill_matches_explicit_elimination():
    rng = np.random.default_rng(0)
    for n, m in ((1, 0), (12, 20), (60, 150), (200, 500)):
        r = rng.integers(0, n, m)
        c = rng.integers(0, n, m)
        for perm in (np.arange(n), rng.permutation(n)):
            f, par = N.symbolic_fill(n, r, c, perm)
            assert f == _fill_by_elimination(n, r, c, perm)
            # every node but the roots has a later parent
            assert all(p == -1 or p > i for i, p in enumerate(par))


def test_amd_is_a_permutation():
    rng = np.random.default_rng(1)
    assert N.amd_order(0, [], []).size == 0
    assert np.array_equal(N.amd_order(1, [], []), [0])
    assert _is_perm(N.amd_order(7, [], []), 7)                # isolated nodes
    for n, m in ((30, 40), (300, 2000), (1000, 3000)):
        r = rng.integers(0, n, m)
        c = rng.integers(0, n, m)
        p1 = N.amd_order(n, r, c)
        assert _is_perm(p1, n)
        # both triangles, duplicates and diagonal entries give the same order
        p2 = N.amd_order(n, np.r_[r, c, r, np.arange(n)], np.r_[c, r, c, np.arange(n)])
        assert np.array_equal(p1, p2)
    with pytest.raises(N.NelsonError):
        N.amd_order(3, [0], [3])


def test_no_fill_where_a_perfect_order_exists():
    rng = np.random.default_rng(2)
    n = 500
    par = np.array([rng.integers(0, i) for i in range(1, n)])  # random tree
    r, c = np.arange(1, n), par
    assert N.symbolic_fill(n, r, c, N.amd_order(n, r, c))[0] == n - 1
    # star: the hub is a dense row and goes last
    r, c = np.zeros(n - 1, np.int32), np.arange(1, n)
    p = N.amd_order(n, r, c)
    assert p[0] == n - 1 and N.symbolic_fill(n, r, c, p)[0] == n - 1
    # clique: every order fills nothing beyond the clique itself
    k = 20
    i, j = np.triu_indices(k, 1)
    assert N.symbolic_fill(k, i, j, N.amd_order(k, i, j))[0] == k * (k - 1) // 2


def test_grid_fill_close_to_exact_minimum_degree():
    n, r, c = _grid(30)
    f_amd = N.symbolic_fill(n, r, c, N.amd_order(n, r, c))[0]
    f_md = N.symbolic_fill(n, r, c, _exact_min_degree(n, r, c))[0]
    f_nat = N.symbolic_fill(n, r, c, np.arange(n))[0]
    cam = np.stack([r, c], 1).ravel()
    pt = np.repeat(np.arange(r.size), 2)
    f_rcm = N.symbolic_fill(n, r, c, N.rcm_order(n, r.size, cam, pt))[0]
    print("grid 30x30 fill: amd", f_amd, "exact md", f_md, "natural", f_nat, "rcm", f_rcm)
    assert f_amd <= 1.1 * f_md
    assert f_amd < 0.4 * f_nat and f_amd < 0.6 * f_rcm
    # the camera-graph entry gives the same order on the same graph
    assert np.array_equal(N.amd_order_camera_graph(n, r.size, cam, pt), N.amd_order(n, r, c))


@pytest.mark.parametrize("scene", ["config0", "grid_shuffled", "config2_small"])
def test_camera_graph_fill_close_to_exact_minimum_degree(scene):
    if scene == "config0":
        p = make_config(0)
        cam, pt, nc, np_ = p.cam_idx, p.pt_idx, p.nc_var, p.np_var
    elif scene == "grid_shuffled":
        p = grid_scene(12, 20, 20000, 2, 8, seed=3)
        inv = np.argsort(np.random.default_rng(1).permutation(p.nc_var)).astype(np.int32)
        cam, pt, nc, np_ = inv[p.cam_idx], p.pt_idx, p.nc_var, p.np_var
    else:
        p = make_config(2, 0.1)
        cam, pt, nc, np_ = p.cam_idx, p.pt_idx, p.nc_var, p.np_var
    r, c = _camera_graph(nc, cam, pt)
    pa = N.amd_order_camera_graph(nc, np_, cam, pt)
    pr = N.rcm_order(nc, np_, cam, pt)
    assert _is_perm(pa, nc)
    fa = N.symbolic_fill(nc, r, c, pa)[0]
    fr = N.symbolic_fill(nc, r, c, pr)[0]
    fn = N.symbolic_fill(nc, r, c, np.arange(nc))[0]
    fm = N.symbolic_fill(nc, r, c, _exact_min_degree(nc, r, c))[0]
    print(scene, "cameras", nc, "fill amd", fa, "exact md", fm, "rcm", fr, "natural", fn)
    assert fa <= 1.05 * fm and fa <= fn
