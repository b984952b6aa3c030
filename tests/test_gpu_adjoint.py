"""Implicit-function adjoint (nl_adjoint) against central finite differences
and against the FP64 CPU reference gradient.

Workload: the differentiable-solve configuration at its stated size (64 ring
cameras with 6-parameter blocks, 5,000 points, k~U{3..8}, about 27.5 k
observations, per-edge weights w~U[0.5,2]); the last two cameras are fixed
nodes so that the solution has no gauge freedom.  LM runs to convergence;
the loss is L = |X_points - X_true|^2.  Gradients w.r.t. observations and
edge weights from nl_adjoint (FP64 and mixed handles) are compared
  * with central differences (h = 1e-6) of the re-converged solution
    (Gauss-Newton steps from the solution, see `converge`) on 200 random
    coordinates, to 1e-4 relative (per coordinate over coordinates whose FD
    magnitude is at least 10% of the largest, and every coordinate against
    the largest);
  * with the oracle's FP64 adjoint (exact Hessian by complex-step derivatives,
    its own Schur solve, the same per-edge VJP) on every coordinate: 1e-8
    (FP64 handle) and 1e-6 (mixed) relative to the gradient's scale.
The adjoint is also driven through a torch.autograd.Function (test harness
only).
"""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import make_config, with_fixed_nodes

pytestmark = pytest.mark.gpu

H = 1e-6
TOL = 1e-4
LM_CONVERGE = dict(maxNumIt=60, maxNumSubIt=10, epsIncSquare=1e-30)
GN_POLISH = dict(maxNumIt=5, epsIncSquare=0.0, epsBVector=0.0, epsChi2=0.0)


def problem():
    p = make_config(4)  # 64 cameras, 5,000 points, weights U[0.5, 2]
    assert (p.nc_var, p.np_var) == (64, 5000)
    return with_fixed_nodes(p, 2, 0)


def converge(g, cams0, pts0, obs, w, lm=True):
    """LM to convergence, then Gauss-Newton steps: near the minimum the cost
    change of a step is below FP64 resolution of chi2, so LM's gain-ratio test
    cannot tell good steps from bad ones; GN steps (no acceptance test, no
    damping: the gauge is fixed) converge to b = 0 at machine precision."""
    g.set_params(cams0, pts0)
    g.set_observations(obs, w)
    if lm:
        g.lm_solve(N.LMSettings(**LM_CONVERGE), trace_cap=0)
    g.gn_solve(N.GNSettings(**GN_POLISH), trace_cap=0)
    return g.get_params()


def fd_gradient(g, p, cams_s, pts_s, coords):
    """Central differences of L at the re-converged solution, warm-started at
    the solution; L(+) - L(-) is formed as sum dX . (X+ + X- - 2 X_true)."""
    xt = p.pts_true[:p.np_var]
    out = []
    for kind, idx in coords:
        vals = []
        for sgn in (+1.0, -1.0):
            obs = p.obs.copy()
            w = p.weight.copy()
            if kind == "obs":
                obs.reshape(-1)[idx] += sgn * H
            else:
                w[idx] += sgn * H
            _, pts = converge(g, cams_s, pts_s, obs, w, lm=False)
            vals.append(pts[:p.np_var].copy())
        xp, xm = vals
        out.append(float(np.sum((xp - xm) * (xp + xm - 2 * xt))) / (2 * H))
    return np.array(out)


@pytest.fixture(scope="module")
def solved():
    p = problem()
    g = N.BAProblemGPU.from_ba(p, precision=N.PREC_FP64)
    cams_s, pts_s = converge(g, p.cams, p.pts, p.obs, p.weight)
    rng = np.random.default_rng(11)
    coords = [("obs", int(i)) for i in rng.choice(2 * p.ne, size=100, replace=False)] + \
             [("w", int(i)) for i in rng.choice(p.ne, size=100, replace=False)]
    fd = fd_gradient(g, p, cams_s, pts_s, coords)
    # restore the converged state
    converge(g, cams_s, pts_s, p.obs, p.weight, lm=False)
    yield p, g, cams_s, pts_s, coords, fd
    g.close()


def _pick(g_obs, g_w, coords):
    return np.array([g_obs.reshape(-1)[i] if k == "obs" else g_w[i] for k, i in coords])


def _check(adj, fd):
    # Per coordinate where the difference quotient is well resolved (at least
    # 10% of the largest): at h = 1e-6 the re-converged solutions carry
    # rounding of about 1e-8 of the gradient scale, which on a coordinate near
    # 1% of the largest is already 1e-4 of its value.  Every coordinate is
    # checked against the scale, and the oracle's independent FP64 adjoint
    # checks every coordinate to 1e-8 (test_adjoint_matches_oracle_adjoint).
    big = np.abs(fd) >= 1e-1 * np.abs(fd).max()
    assert big.sum() >= 5
    rel = np.abs(adj[big] - fd[big]) / np.abs(fd[big])
    assert rel.max() <= TOL, (rel.max(), np.argmax(rel))
    assert np.abs(adj - fd).max() <= TOL * np.abs(fd).max()


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_adjoint_matches_finite_differences(solved, prec):
    p, g64, cams_s, pts_s, coords, fd = solved
    g = g64 if prec == N.PREC_FP64 else N.BAProblemGPU.from_ba(p, precision=prec)
    g.set_params(cams_s, pts_s)
    g.set_observations(p.obs, p.weight)
    dL = 2.0 * (pts_s[:p.np_var] - p.pts_true[:p.np_var])
    g_obs, g_w, rep = g.adjoint(dL_dpts=dL, sweeps=4)
    print(rep)
    assert rep["ok"] == 1
    assert rep["residual_norm"] <= 1e-6 * rep["grad_norm"]
    _check(_pick(g_obs, g_w, coords), fd)
    if g is not g64:
        g.close()


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_adjoint_refinement_converges(solved, prec):
    """|dL/dx - H mu| falls with the refinement rounds to a floor far below
    the gradient (the FP32 factor of the mixed handle only preconditions)."""
    p, g64, cams_s, pts_s, coords, fd = solved
    g = g64 if prec == N.PREC_FP64 else N.BAProblemGPU.from_ba(p, precision=prec)
    g.set_params(cams_s, pts_s)
    g.set_observations(p.obs, p.weight)
    dL = 2.0 * (pts_s[:p.np_var] - p.pts_true[:p.np_var])
    res = [g.adjoint(dL_dpts=dL, sweeps=s)[2]["residual_norm"] for s in range(7)]
    gn = np.linalg.norm(dL)
    print(prec, [r / gn for r in res])
    assert res[1] < 0.1 * res[0]
    assert min(res) <= 1e-6 * gn
    if g is not g64:
        g.close()


@pytest.mark.parametrize("prec,tol", [(N.PREC_FP64, 1e-8), (N.PREC_MIXED, 1e-6)])
def test_adjoint_matches_oracle_adjoint(solved, oracle_lib, prec, tol):
    """FP64 CPU reference gradient: the oracle's adjoint at the same converged
    parameters, compared on every observation and weight coordinate and on mu."""
    p, g64, cams_s, pts_s, coords, fd = solved
    g = g64 if prec == N.PREC_FP64 else N.BAProblemGPU.from_ba(p, precision=prec)
    g.set_params(cams_s, pts_s)
    g.set_observations(p.obs, p.weight)
    dL = 2.0 * (pts_s[:p.np_var] - p.pts_true[:p.np_var])
    g_obs, g_w, rep, mu_c, mu_p = g.adjoint(dL_dpts=dL, sweeps=4, want_mu=True)
    q = problem()
    q.cams, q.pts = cams_s.copy(), pts_s.copy()
    o = oracle_lib.Oracle.from_ba(q)
    o_obs, o_w, o_mc, o_mp = o.adjoint(dL_dpts=dL)
    for a, b in ((g_obs, o_obs), (g_w, o_w), (mu_p, o_mp), (mu_c, o_mc)):
        assert np.abs(a - b).max() <= tol * np.abs(b).max(), (np.abs(a - b).max(), np.abs(b).max())
    # the oracle's gradient agrees with the finite differences too
    _check(_pick(o_obs, o_w, coords), fd)
    if g is not g64:
        g.close()


def test_adjoint_through_autograd(solved):
    """A torch.autograd.Function over the C ABI: forward = LM to convergence,
    backward = nl_adjoint.  obs.grad / weight.grad equal nl_adjoint's output."""
    import torch
    p, g, cams_s, pts_s, coords, fd = solved

    class BASolve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, obs, w):
            _, pts = converge(g, cams_s, pts_s, obs.detach().numpy(), w.detach().numpy(), lm=False)
            return torch.from_numpy(pts[:p.np_var].copy())

        @staticmethod
        def backward(ctx, grad_pts):
            g_obs, g_w, _ = g.adjoint(dL_dpts=grad_pts.detach().numpy(), sweeps=4)
            return torch.from_numpy(g_obs), torch.from_numpy(g_w)

    obs = torch.tensor(p.obs, dtype=torch.float64, requires_grad=True)
    w = torch.tensor(p.weight, dtype=torch.float64, requires_grad=True)
    X = BASolve.apply(obs, w)
    L = ((X - torch.from_numpy(p.pts_true[:p.np_var])) ** 2).sum()
    L.backward()
    adj = _pick(obs.grad.numpy(), w.grad.numpy(), coords)
    _check(adj, fd)


def test_adjoint_requires_ready_and_valid_sweeps():
    p = problem()
    g = N.BAProblemGPU(p.bc, p.nc_var, p.np_var, p.nc_fix, p.np_fix, precision=N.PREC_FP64)
    with pytest.raises(N.NelsonError):
        g.adjoint(dL_dpts=np.zeros((p.np_var, 3)))  # structure not ready
    g.close()
