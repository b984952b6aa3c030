"""Pins the FP64 CPU oracle against the reference's own known-answer tests.

The reference (a C++/Eigen library) ships no golden vectors; its tests check
(1) the 5x2D / 3x3D identity-Jacobian fixture, which GN and LM must drive
to chi2 < 1e-12 from uniform noise of 0.5 (nelson/tests/testDoubleSectionCommon.hpp:58-130,
testDoubleSectionSchurCommon.hpp:60-115), with random and AMD permutations
(testDoubleSectionSchurDiagBlockWWtFFFF.cpp:482-504); (2) the 3x5 W pattern
and its S = U - W W' pattern (testMatrixWWtMultiplier.cpp:36-59) and the
multiplier identities at dummy_precision (1e-12).  These tests restate those
checks against the oracle.
"""
import numpy as np
import pytest

from nelson_b200.problems import (EDGE_BINARY_UU, EDGE_BINARY_UV, EDGE_UNARY_U, EDGE_UNARY_V,
                                  LinearEdge, LinearProblem, add_uniform_noise, make_config,
                                  points2d3d_fixture)

DUMMY_PRECISION = 1e-12  # Eigen::NumTraits<double>::dummy_precision()


def _variants():
    for ubd in (False, True):
        for wbd in (False, True):
            yield ubd, wbd


@pytest.mark.parametrize("ubd,wbd", list(_variants()))
@pytest.mark.parametrize("algo", ["gn", "lm"])
@pytest.mark.parametrize("perm", ["standard", "permute", "reverse"])
def test_points2d3d_fixture_converges(oracle_lib, ubd, wbd, algo, perm):
    O = oracle_lib.Oracle
    lp = points2d3d_fixture(seed=11, u_block_diagonal=ubd, w_block_diagonal=wbd)
    pm = None
    if perm == "permute":
        pm = np.random.default_rng(3).permutation(5)
    elif perm == "reverse":
        pm = np.arange(5)[::-1].copy()
    o = O.from_linear(lp, perm=pm)
    # chi2 is zero at the ground truth (testDoubleSectionCommon.hpp:58)
    assert o.update(True) == 0.0
    rng = np.random.default_rng(5)
    for rep in range(3):  # the reference adds noise again before each solver variant
        add_uniform_noise(lp, 0.5, rng)
        o.set_params(lp.u, lp.v)
        assert o.update(False) > 1e-3
        if algo == "gn":
            reason, tr, it = o.gn_solve()
        else:
            reason, tr, it, sub = o.lm_solve()
        assert reason.startswith("Success"), reason
        assert o.chi2() < DUMMY_PRECISION


def _wwt_problem():
    """U: 3 blocks of size 6 (diagonal + block (0, 2)), V: 5 blocks of size 3,
    W pattern of testMatrixWWtMultiplier.cpp:36-42 (row 2 without (2,3), (2,4))."""
    rng = np.random.default_rng(21)
    bu, bv = 6, 3
    wpat = [(0, 0), (0, 3), (0, 4), (1, 0), (1, 1), (1, 3), (2, 1), (2, 2)]
    edges = []
    for i in range(3):
        edges.append(LinearEdge(EDGE_UNARY_U, i, -1, rng.normal(size=(3, bu)) * 0 + np.eye(3, bu) * 2, None,
                                rng.normal(size=3)))
        edges.append(LinearEdge(EDGE_UNARY_U, i, -1, np.roll(np.eye(3, bu), 3, axis=1) * 2, None,
                                rng.normal(size=3)))
    for j in range(5):
        edges.append(LinearEdge(EDGE_UNARY_V, j, -1, np.eye(3) * 3, None, rng.normal(size=3)))
    edges.append(LinearEdge(EDGE_BINARY_UU, 0, 2, rng.normal(size=(3, bu)), rng.normal(size=(3, bu)),
                            rng.normal(size=3)))
    for (i, j) in wpat:
        edges.append(LinearEdge(EDGE_BINARY_UV, i, j, rng.normal(size=(3, bu)), rng.normal(size=(3, bv)),
                                rng.normal(size=3)))
    lp = LinearProblem(bu=bu, bv=bv, u=rng.normal(size=(3, bu)), v=rng.normal(size=(5, bv)), nu_var=3, nv_var=5,
                       edges=edges)
    return lp, wpat


def _dense(o, U, V, W, uR, vR, wR):
    bu, bv = o.bu, o.bv
    nu, nv = o.nu_var, o.nv_var
    Ud = np.zeros((nu * bu, nu * bu))
    for q, (r, c) in enumerate(uR):
        Ud[r * bu:(r + 1) * bu, c * bu:(c + 1) * bu] = U[q]
        if r != c:
            Ud[c * bu:(c + 1) * bu, r * bu:(r + 1) * bu] = U[q].T
    Vd = np.zeros((nv * bv, nv * bv))
    for q, (r, c) in enumerate(vR):
        Vd[r * bv:(r + 1) * bv, c * bv:(c + 1) * bv] = V[q]
    Wd = np.zeros((nu * bu, nv * bv))
    for q, (r, c) in enumerate(wR):
        Wd[r * bu:(r + 1) * bu, c * bv:(c + 1) * bv] = W[q]
    return Ud, Vd, Wd


def test_wwt_pattern_and_values(oracle_lib):
    lp, wpat = _wwt_problem()
    o = oracle_lib.Oracle.from_linear(lp)
    uR, vR, wR = o.patterns()
    # W UIDs follow CSR order of the pattern (DoubleSection.hpp:181-191)
    assert [tuple(x) for x in wR] == sorted(wpat)
    # U UIDs follow CSC order of the upper pattern: (0,0) (1,1) (0,2) (2,2)
    assert [tuple(x) for x in uR] == [(0, 0), (1, 1), (0, 2), (2, 2)]
    o.update(True)
    ok = o.compute_increment(0.0, 0.0)
    assert ok
    S, bS = o.schur()
    # expected upper block pattern (testMatrixWWtMultiplier.cpp:56-59, plus U(0,2))
    #   X X X      (0,2) comes from U here
    #     X X
    #       X
    nz = np.array([[np.abs(S[i * 6:(i + 1) * 6, j * 6:(j + 1) * 6]).max() > 0 for j in range(3)] for i in range(3)])
    assert (nz == np.array([[1, 1, 1], [0, 1, 1], [0, 0, 1]], bool)).all()
    U, V, W, bU, bV = o.hessian()
    Ud, Vd, Wd = _dense(o, U, V, W, uR, vR, wR)
    Sref = np.triu(Ud - Wd @ np.linalg.inv(Vd) @ Wd.T)
    assert np.abs(np.triu(S) - Sref).max() < DUMMY_PRECISION * max(1.0, np.abs(Sref).max())
    # WtX / Vinv identities: the increment solves the full system
    H = np.block([[Ud, Wd], [Wd.T, Vd]])
    x = np.linalg.solve(H, -np.concatenate([bU, bV]))
    du, dv = o.increment()
    assert np.abs(np.concatenate([du, dv]) - x).max() < 1e-10 * max(1.0, np.abs(x).max())


@pytest.mark.parametrize("damp", [1e-2, 1.0, 10.0])
def test_ba_schur_increment_matches_dense_solve(oracle_lib, damp):
    p = make_config(0, 0.3)
    o = oracle_lib.Oracle.from_ba(p)
    o.update(True)
    U, V, W, bU, bV = o.hessian()
    uR, vR, wR = o.patterns()
    Ud, Vd, Wd = _dense(o, U, V, W, uR, vR, wR)
    mu = damp * o.max_abs_hdiag() * 1e-3  # LM damping levels (tau = 1e-3)
    H = np.block([[Ud, Wd], [Wd.T, Vd]]) + mu * np.eye(Ud.shape[0] + Vd.shape[0])
    x = np.linalg.solve(H, -np.concatenate([bU, bV]))
    assert o.compute_increment(0.0, mu)
    du, dv = o.increment()
    assert np.abs(np.concatenate([du, dv]) - x).max() < 1e-9 * np.abs(x).max()


def test_relative_damping_matches_reference_formula(oracle_lib):
    """diag(S) += rel diag(U) + abs and V scaled by (1 + rel) + abs
    (SolverCholeskySchur.hpp:121-124, MatrixDiagInv.hpp:37-40)."""
    p = make_config(0, 0.2)
    o = oracle_lib.Oracle.from_ba(p)
    o.update(True)
    U, V, W, bU, bV = o.hessian()
    uR, vR, wR = o.patterns()
    Ud, Vd, Wd = _dense(o, U, V, W, uR, vR, wR)
    rel, ab = 0.3, 2.0
    Vd2 = Vd + np.diag(np.diag(Vd) * rel + ab)
    S = Ud - Wd @ np.linalg.inv(Vd2) @ Wd.T
    S = S + np.diag(rel * np.diag(Ud) + ab)
    assert o.compute_increment(rel, ab)
    So, bSo = o.schur()
    assert np.abs(np.triu(So) - np.triu(S)).max() < 1e-9 * np.abs(S).max()


def test_uid_maps_reference_order(oracle_lib):
    p = make_config(0, 0.2)
    perm = np.random.default_rng(9).permutation(p.nc_var)
    o = oracle_lib.Oracle.from_ba(p, perm=perm)
    uR, vR, wR = o.patterns()
    h11, h12, h22 = o.edge_uids()
    # U / V diagonal, UIDs ascending with the (internal) index
    assert (uR[:, 0] == uR[:, 1]).all() and (np.diff(uR[:, 1]) > 0).all()
    assert (vR[:, 0] == vR[:, 1]).all() and (np.diff(vR[:, 1]) > 0).all()
    # W in CSR order over permuted cameras
    key = wR[:, 0].astype(np.int64) * p.np_var + wR[:, 1]
    assert (np.diff(key) > 0).all()
    # each edge's UIDs point at its own blocks
    assert (uR[h11, 0] == perm[p.cam_idx]).all()
    assert (vR[h22, 0] == p.pt_idx).all()
    assert (wR[h12, 0] == perm[p.cam_idx]).all() and (wR[h12, 1] == p.pt_idx).all()


def test_fixed_nodes_drop_blocks(oracle_lib):
    p = make_config(0, 0.2)
    # camera 0 and point 0 become fixed nodes, as in BASchurPerfomances.cpp:103-153
    cams, pts = p.cams, p.pts
    p.cam_fixed = (p.cam_idx == 0).astype(np.int32)
    p.pt_fixed = (p.pt_idx == 0).astype(np.int32)
    p.cam_idx = np.where(p.cam_fixed == 1, 0, p.cam_idx - 1).astype(np.int32)
    p.pt_idx = np.where(p.pt_fixed == 1, 0, p.pt_idx - 1).astype(np.int32)
    p.cams = np.concatenate([cams[1:], cams[:1]])
    p.pts = np.concatenate([pts[1:], pts[:1]])
    p.nc_var -= 1
    p.np_var -= 1
    p.nc_fix = p.np_fix = 1
    o = oracle_lib.Oracle.from_ba(p)
    h11, h12, h22 = o.edge_uids()
    assert (h11[p.cam_fixed == 1] == -1).all() and (h12[(p.cam_fixed == 1) | (p.pt_fixed == 1)] == -1).all()
    assert (h22[p.pt_fixed == 1] == -1).all()
    reason, tr, it, sub = o.lm_solve(oracle_lib.LMSettings(maxNumIt=15))
    assert tr[-1, 2] < tr[0, 2]


def test_lm_trace_follows_reference_rules(oracle_lib):
    p = make_config(0)
    o = oracle_lib.Oracle.from_ba(p)
    s = oracle_lib.LMSettings(maxNumIt=10)
    reason, tr, it, sub = o.lm_solve(s)
    assert reason == "MaxIterationReached" and it == 10
    assert tr[0, 0] == -1 and tr[0, 1] == -1
    mu = tr[1, 3]
    for k in range(1, len(tr) - 1):
        rho, acc = tr[k, 4], tr[k, 7]
        nxt = tr[k + 1, 3]
        if acc:  # mu *= clamp(1 - (2 rho - 1)^3, 1/3, 2/3)
            a = min(2 / 3, max(1 / 3, 1 - (2 * rho - 1) ** 3))
            assert nxt == pytest.approx(tr[k, 3] * a, rel=1e-12)
        else:
            assert nxt > tr[k, 3]
    assert tr[-1, 2] < 0.1 * tr[0, 2]


def test_dense_cholesky(oracle_lib):
    rng = np.random.default_rng(0)
    n = 300
    A = rng.normal(size=(n, n))
    A = A @ A.T + n * np.eye(n)
    L = A.copy()
    assert oracle_lib.dense_cholesky(L, threads=2)
    L = np.tril(L)
    assert np.abs(L @ L.T - A).max() < 1e-10 * np.abs(A).max()
    B = -np.eye(4)
    assert not oracle_lib.dense_cholesky(B)


def test_oracle_adjoint_matches_finite_differences():
    """The oracle's FP64 implicit-function adjoint (exact Hessian by
    complex-step derivatives) against central differences (h = 1e-6) of the
    oracle's own re-converged solution, on a small weighted ring scene with
    two fixed cameras (no gauge freedom): 1e-4 relative."""
    import numpy as np

    from nelson_b200.problems import ring_scene, with_fixed_nodes
    from oracle.oracle import GNSettings, LMSettings, Oracle

    def scene():
        return with_fixed_nodes(ring_scene(10, 150, 3, 8, 6, seed=99, name="adj", weights=True), 2, 0)

    gn = dict(maxNumIt=6, epsIncSquare=0.0, epsBVector=0.0, epsChi2=0.0)
    p = scene()
    o = Oracle.from_ba(p)
    o.lm_solve(LMSettings(maxNumIt=60))
    o.gn_solve(GNSettings(**gn))
    cams_s, pts_s = o.get_params()
    xt = p.pts_true[:p.np_var]
    g_obs, g_w, _, _ = o.adjoint(dL_dpts=2.0 * (pts_s[:p.np_var] - xt))
    rng = np.random.default_rng(0)
    coords = [("obs", int(i)) for i in rng.choice(2 * p.ne, 12, replace=False)] + \
             [("w", int(i)) for i in rng.choice(p.ne, 12, replace=False)]
    h = 1e-6
    adjs, fds = [], []
    for kind, idx in coords:
        vals = []
        for sgn in (1.0, -1.0):
            q = scene()
            q.cams, q.pts = cams_s.copy(), pts_s.copy()
            if kind == "obs":
                q.obs.reshape(-1)[idx] += sgn * h
            else:
                q.weight[idx] += sgn * h
            oo = Oracle.from_ba(q)
            oo.gn_solve(GNSettings(**gn))
            vals.append(oo.get_params()[1][:p.np_var].copy())
        xp, xm = vals
        fd = float(np.sum((xp - xm) * (xp + xm - 2 * xt))) / (2 * h)
        adjs.append(g_obs.reshape(-1)[idx] if kind == "obs" else g_w[idx])
        fds.append(fd)
    adjs, fds = np.array(adjs), np.array(fds)
    # per coordinate where the difference quotient is well above its noise
    # (|fd| >= 1% of the largest), and every coordinate against the scale
    big = np.abs(fds) >= 1e-2 * np.abs(fds).max()
    assert big.sum() >= 10
    assert (np.abs(adjs[big] - fds[big]) <= 1e-4 * np.abs(fds[big])).all(), (adjs, fds)
    assert np.abs(adjs - fds).max() <= 1e-4 * np.abs(fds).max()


def test_handle_passes_as_a_full_pointer(oracle_lib):
    """The oracle handle stays a pointer object: its entry points without
    declared argument types would otherwise receive a 32-bit C int and lose
    the upper half of a heap address above 4 GB."""
    import ctypes
    o = oracle_lib.Oracle.from_ba(make_config(0))
    assert isinstance(o.h, ctypes.c_void_p) and o.h.value
    o.update(True)
    assert o.chi2() > 0
