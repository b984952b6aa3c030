"""The reverse Cuthill-McKee camera order (nl_rcm_order, the host function
behind nl_permute_rcm_u) on the CPU: on a camera-shuffled aerial grid it
gives back a narrow band of co-observing camera pairs, as scipy's RCM does
on the same graph, and it is always a permutation."""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import reverse_cuthill_mckee

from nelson_b200 import native as N
from nelson_b200.problems import grid_scene


def _camera_graph(nc, cam, pt):
    """Cameras that share a point."""
    order = np.argsort(pt, kind="stable")
    cam, pt = cam[order], pt[order]
    rows, cols = [], []
    starts = np.flatnonzero(np.r_[True, pt[1:] != pt[:-1]])
    ends = np.r_[starts[1:], pt.size]
    for a, b in zip(starts, ends):
        c = np.unique(cam[a:b])
        i, j = np.meshgrid(c, c, indexing="ij")
        rows.append(i.ravel())
        cols.append(j.ravel())
    r, c = np.concatenate(rows), np.concatenate(cols)
    return sp.coo_matrix((np.ones(r.size), (r, c)), shape=(nc, nc)).tocsr()


def _bandwidth(G, pos):
    G = G.tocoo()
    return int(np.abs(pos[G.row] - pos[G.col]).max())


def _profile(G, pos):
    """Sum over positions of the distance to the row's first neighbour: the
    size of the envelope an envelope Cholesky works on."""
    G = G.tocsr()
    first = np.array([pos[G.indices[G.indptr[i]:G.indptr[i + 1]]].min() for i in range(G.shape[0])])
    return int((pos - first).sum())


def test_rcm_restores_the_band_of_a_shuffled_grid():
    p = grid_scene(12, 20, 20000, 2, 8, seed=3)  # cameras within two grid cells see each point
    rng = np.random.default_rng(1)
    q = rng.permutation(p.nc_var)
    inv = np.argsort(q).astype(np.int32)
    cam = inv[p.cam_idx]                  # the same scene, cameras in a random order
    G = _camera_graph(p.nc_var, cam, p.pt_idx)
    perm = N.rcm_order(p.nc_var, p.np_var, cam, p.pt_idx)
    assert np.array_equal(np.sort(perm), np.arange(p.nc_var))
    sci = reverse_cuthill_mckee(G, symmetric_mode=True)
    sci_pos = np.empty(p.nc_var, np.int64)
    sci_pos[sci] = np.arange(p.nc_var)
    ident = np.arange(p.nc_var)
    natural_graph = _camera_graph(p.nc_var, p.cam_idx, p.pt_idx)
    # the envelope: below half of the shuffled order's, no larger than the
    # grid's own order, within 10% of scipy's RCM on the same graph
    ours = _profile(G, perm)
    assert ours < 0.5 * _profile(G, ident), (ours, _profile(G, ident))
    assert ours <= _profile(natural_graph, ident)
    assert ours <= 1.1 * _profile(G, sci_pos), (ours, _profile(G, sci_pos))
    assert _bandwidth(G, perm) <= 1.1 * _bandwidth(G, sci_pos)


def test_rcm_handles_disconnected_and_isolated_cameras():
    # two separate chains and a camera that sees nothing
    cam = np.array([0, 1, 1, 2, 4, 5], np.int32)
    pt = np.array([0, 0, 1, 1, 2, 2], np.int32)
    perm = N.rcm_order(7, 3, cam, pt)
    assert np.array_equal(np.sort(perm), np.arange(7))
    # each chain stays contiguous
    for chain in ([0, 1, 2], [4, 5]):
        pos = np.sort(perm[chain])
        assert pos[-1] - pos[0] == len(chain) - 1


def test_rcm_rejects_bad_edges():
    with pytest.raises(N.NelsonError):
        N.rcm_order(3, 2, np.array([0, 3], np.int32), np.array([0, 1], np.int32))
    with pytest.raises(N.NelsonError):
        N.rcm_order(3, 2, np.array([0, 1], np.int32), np.array([0, 2], np.int32))
