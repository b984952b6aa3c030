"""Unrolled differentiation through 10 LM steps (nl_unroll_record /
nl_unroll_adjoint) against central finite differences.

Workload: the differentiable-solve configuration at its stated size (64 ring
cameras with 6-parameter blocks, 5,000 points, k~U{3..8}, per-edge weights
w~U[0.5,2], the last two cameras fixed).  LevenbergMarquardt runs 10
iterations from the perturbed start; the damping of its accepted steps is the
schedule of the unrolled map x_0 -> x_10 (the accept / reject choices and the
damping updates are held fixed).  The loss is L = |X_10 - X_true|^2.

* The replayed record reproduces the LM run (same kernels, same order).
* Gradients w.r.t. observations, edge weights, the initial camera parameters
  (axis-angle, t) and the initial points, from the FP64 and the mixed handles,
  against finite differences of the FP64 replay on 200 random coordinates
  (50 per group), to 1e-4 relative plus an absolute floor (`_check`).  The
  difference is central and Richardson-extrapolated, D = (4 D(h/2) - D(h)) / 3
  with h = 1e-3 (truncation O(h^4)).  A plain central difference at a small
  step is rounding-limited here: the last of the 10 steps are damped by
  mu ~ 0.2 only, and on the largest observation coordinate the oracle's replay
  gives -0.20245428, -0.20245414 and -0.20245553 at h = 1e-3, 1e-4 and 1e-5,
  -0.20242395 at h = 1e-6 and -0.20230839 at h = 1e-7, while the adjoint
  gives -0.20245431: the quotient's rounding noise is about 1.7e-11 / h.
* The mixed handle follows the FP64 map: each recorded step's increment from
  the FP32 Hessian is refined against (J'WJ + mu I) delta = -J'W r in FP64,
  and so is each step adjoint u = A^-1 a (the FP32 factor preconditions).
* A few coordinates against the same difference taken with the FP64 CPU
  oracle's own replay (update(true), computeIncrement(0, mu_k), oplus).
"""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import make_config, with_fixed_nodes

pytestmark = pytest.mark.gpu

H = 1e-3          # Richardson pair h, h / 2
TOL = 1e-4
ATOL = 1e-7       # about 3x the rounding noise of the extrapolated quotient
K_ITERS = 10


def problem():
    p = make_config(4)
    return with_fixed_nodes(p, 2, 0)


def accepted_mus(tr):
    return [float(r[3]) for r in tr if r[0] >= 0 and r[7] == 1]


def loss_diff(xp, xm, xt):
    return float(np.sum((xp - xm) * (xp + xm - 2 * xt)))


def richardson(d):
    """(4 D(H/2) - D(H)) / 3 for the central difference D(h)."""
    return (4.0 * d(H / 2) - d(H)) / 3.0


@pytest.fixture(scope="module")
def unrolled():
    p = problem()
    g = N.BAProblemGPU.from_ba(p, precision=N.PREC_FP64)
    _, tr, its, _ = g.lm_solve(N.LMSettings(maxNumIt=K_ITERS))
    x_lm = g.get_params()
    mus = accepted_mus(tr)
    assert len(mus) == K_ITERS
    xt = p.pts_true[:p.np_var]

    def replay(cams, pts, obs, w):
        g.set_params(cams, pts)
        g.set_observations(obs, w)
        g.unroll_record(mus)
        return g.get_params()[1][:p.np_var].copy()

    rng = np.random.default_rng(21)
    ncv = p.nc_var
    coords = [("obs", int(i)) for i in rng.choice(2 * p.ne, 50, replace=False)] + \
             [("w", int(i)) for i in rng.choice(p.ne, 50, replace=False)] + \
             [("cam", int(i)) for i in rng.choice(ncv * p.bc, 50, replace=False)] + \
             [("pt", int(i)) for i in rng.choice(3 * p.np_var, 50, replace=False)]
    def central(kind, idx, h):
        xs = []
        for sgn in (1.0, -1.0):
            cams, pts, obs, w = p.cams.copy(), p.pts.copy(), p.obs.copy(), p.weight.copy()
            if kind == "obs":
                obs.reshape(-1)[idx] += sgn * h
            elif kind == "w":
                w[idx] += sgn * h
            elif kind == "cam":
                cams[:ncv].reshape(-1)[idx] += sgn * h
            else:
                pts[:p.np_var].reshape(-1)[idx] += sgn * h
            xs.append(replay(cams, pts, obs, w))
        return loss_diff(xs[0], xs[1], xt) / (2 * h)

    fd = [richardson(lambda h: central(kind, idx, h)) for kind, idx in coords]
    g.set_observations(p.obs, p.weight)
    yield p, g, mus, x_lm, coords, np.array(fd)
    g.close()


def _pick(g_obs, g_w, g_c, g_p, p, coords):
    out = []
    for kind, idx in coords:
        if kind == "obs":
            out.append(g_obs.reshape(-1)[idx])
        elif kind == "w":
            out.append(g_w[idx])
        elif kind == "cam":
            out.append(g_c.reshape(-1)[idx])
        else:
            out.append(g_p.reshape(-1)[idx])
    return np.array(out)


def _check(adj, fd, coords):
    """Per coordinate |adj - fd| <= 1e-4 |fd| + 1e-7.  The absolute part covers
    the extrapolated quotient's rounding noise (about 5e-8: 1.7e-11 / h at
    h = 5e-4 and 1e-3, combined with weights 4/3 and 1/3), which matters for
    the coordinates whose gradient is small, e.g. the initial cameras' after
    10 steps (largest 0.011)."""
    kinds = np.array([k for k, _ in coords])
    for kind in ("obs", "w", "cam", "pt"):
        m = kinds == kind
        a, f = adj[m], fd[m]
        scale = np.abs(f).max()
        err = np.abs(a - f)
        big = np.abs(f) >= 1e-2 * scale
        print(kind, "scale", scale, "max rel (|fd| >= 1% of scale)", (err[big] / np.abs(f[big])).max(),
              "max abs", err.max())
        assert (err <= TOL * np.abs(f) + ATOL).all(), (kind, (err / (TOL * np.abs(f) + ATOL)).max())


def test_replay_reproduces_lm(unrolled):
    p, g, mus, x_lm, coords, fd = unrolled
    g.set_params(p.cams, p.pts)
    rep = g.unroll_record(mus)
    assert rep["ok"] == 1 and rep["steps"] == K_ITERS
    cams, pts = g.get_params()
    assert np.array_equal(pts, x_lm[1]) and np.array_equal(cams, x_lm[0])


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_unrolled_gradient_matches_finite_differences(unrolled, prec):
    p, g64, mus, x_lm, coords, fd = unrolled
    g = g64 if prec == N.PREC_FP64 else N.BAProblemGPU.from_ba(p, precision=prec)
    g.set_params(p.cams, p.pts)
    g.set_observations(p.obs, p.weight)
    rep = g.unroll_record(mus)
    assert rep["ok"] == 1
    xK = g.get_params()[1][:p.np_var]
    dL = 2.0 * (xK - p.pts_true[:p.np_var])
    g_obs, g_w, g_c, g_p, rep = g.unroll_adjoint(dL_dpts=dL)
    assert rep["ok"] == 1 and rep["steps"] == K_ITERS
    print(prec, "adjoint device ms", rep["device_ms"])
    _check(_pick(g_obs, g_w, g_c, g_p, p, coords), fd, coords)
    # the parameters are back at x_K
    assert np.array_equal(g.get_params()[1][:p.np_var], xK)
    if g is not g64:
        g.close()


def test_unrolled_zero_steps_passes_the_loss_gradient(unrolled):
    """K = 0: x_K = x_0, so dL/dx_0 = dL/dx_K (points; cameras through the
    axis-angle Jacobian) and the data gradients vanish."""
    p, g, mus, x_lm, coords, fd = unrolled
    g.set_params(p.cams, p.pts)
    g.unroll_record([])
    dL = np.random.default_rng(3).normal(size=(p.np_var, 3))
    g_obs, g_w, g_c, g_p, _ = g.unroll_adjoint(dL_dpts=dL)
    assert np.array_equal(g_p, dL)
    assert not g_obs.any() and not g_w.any() and not g_c.any()


def test_unrolled_matches_cpu_oracle_replay(unrolled, oracle_lib):
    """FP64 CPU reference: the oracle replays the same schedule (its own
    update / computeIncrement(0, mu_k) / oplus); its x_10 equals the GPU's to
    1e-8 and its central differences agree with the GPU adjoint on the
    largest coordinates of each group."""
    p, g, mus, x_lm, coords, fd = unrolled

    def oracle_replay(q):
        o = oracle_lib.Oracle.from_ba(q)
        for mu in mus:
            o.update(True)
            assert o.compute_increment(0.0, mu)
            o.oplus()
        return o.get_params()[1][:p.np_var].copy()

    x_o = oracle_replay(problem())
    assert np.abs(x_o - x_lm[1][:p.np_var]).max() <= 1e-8 * np.abs(x_o).max()
    g.set_params(p.cams, p.pts)
    g.unroll_record(mus)
    xK = g.get_params()[1][:p.np_var]
    g_obs, g_w, g_c, g_p, _ = g.unroll_adjoint(dL_dpts=2.0 * (xK - p.pts_true[:p.np_var]))
    adj = _pick(g_obs, g_w, g_c, g_p, p, coords)
    xt = p.pts_true[:p.np_var]
    kinds = np.array([k for k, _ in coords])
    for kind in ("obs", "w", "cam", "pt"):
        j = int(np.flatnonzero(kinds == kind)[np.argmax(np.abs(fd[kinds == kind]))])
        _, idx = coords[j]

        def central(h):
            xs = []
            for sgn in (1.0, -1.0):
                q = problem()
                if kind == "obs":
                    q.obs.reshape(-1)[idx] += sgn * h
                elif kind == "w":
                    q.weight[idx] += sgn * h
                elif kind == "cam":
                    q.cams[:p.nc_var].reshape(-1)[idx] += sgn * h
                else:
                    q.pts[:p.np_var].reshape(-1)[idx] += sgn * h
                xs.append(oracle_replay(q))
            return loss_diff(xs[0], xs[1], xt) / (2 * h)

        cpu = richardson(central)
        assert abs(adj[j] - cpu) <= TOL * abs(cpu) + ATOL, (kind, idx, adj[j], cpu)
