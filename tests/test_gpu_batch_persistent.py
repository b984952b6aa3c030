"""Many uneven problems in one persistent launch (nl_batch_*).

Problems from the batched configuration's generator (6-parameter cameras
U{8..64}, points U{200..4000}, k~U{3..8}), plus problems with fixed cameras /
points and duplicate edges.  The launch's CTAs take problems from a device
work queue and solve each one's whole LM in FP64.

* every problem against the FP64 oracle's LM on the same problem: final cost
  to 1e-9, the same termination reason and iteration count, points to 1e-6;
* the results do not depend on the launch shape (threads per CTA, CTAs per
  SM) or on the other problems of the batch: bit-identical;
* the autotuner returns a valid launch shape and changes no result.
"""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import BAProblem, make_batch, ring_scene, with_fixed_nodes

pytestmark = pytest.mark.gpu

SET = dict(maxNumIt=8)


def _extra_problems():
    a = with_fixed_nodes(ring_scene(12, 300, 3, 8, 6, seed=77, name="fixed"), 2, 5)
    p = ring_scene(10, 250, 3, 8, 6, seed=78, name="dup")
    rng = np.random.default_rng(5)
    idx = rng.choice(p.ne, size=40, replace=False)
    d = BAProblem(bc=p.bc, cams=p.cams, pts=p.pts, nc_var=p.nc_var, np_var=p.np_var,
                  cam_idx=np.concatenate([p.cam_idx, p.cam_idx[idx]]).astype(np.int32),
                  pt_idx=np.concatenate([p.pt_idx, p.pt_idx[idx]]).astype(np.int32),
                  obs=np.concatenate([p.obs, p.obs[idx] + rng.normal(0, 0.3, size=(40, 2))]), f=p.f, cx=p.cx,
                  cy=p.cy, name="dup")
    w = ring_scene(9, 220, 3, 8, 6, seed=79, name="weighted", weights=True)
    return [a, d, w]


@pytest.fixture(scope="module")
def probs():
    return make_batch(20) + _extra_problems()


def _solve(problems, **kw):
    hs = [N.BAProblemGPU.from_ba(p, precision=N.PREC_FP64) for p in problems]
    b = N.PersistentBatch(hs)
    out = b.lm_solve(N.LMSettings(**SET), **kw)
    params = [g.get_params() for g in hs]
    b.close()
    for g in hs:
        g.close()
    return out, params


def test_batch_matches_oracle(probs, oracle_lib):
    (reasons, chi2, its, lat, solve_ms, dev_ms), params = _solve(probs)
    assert dev_ms > 0 and (lat > 0).all() and (solve_ms > 0).all()
    for k, p in enumerate(probs):
        o = oracle_lib.Oracle.from_ba(p)
        r_o, _, it_o, _ = o.lm_solve(oracle_lib.LMSettings(**SET))
        assert chi2[k] == pytest.approx(o.chi2(), rel=1e-9), (k, p.name)
        # at convergence |inc|^2 can cross epsIncSquare in one and not the
        # other (rounding): then the last iterations differ, the cost does not
        if reasons[k] == r_o:
            assert its[k] == it_o, (k, p.name)
        else:
            assert {reasons[k], r_o} <= {"SuccessSmallIncrement", "MaxIterationReached"}, (k, p.name)
        pts_o = o.get_params()[1]
        assert np.abs(params[k][1] - pts_o).max() <= 1e-6 * np.abs(pts_o).max(), (k, p.name)


def test_results_independent_of_launch_shape_and_batch(probs):
    (_, chi2_a, _, _, _, _), pa = _solve(probs, threads=256, ctas_per_sm=1)
    for nt, cps in ((128, 2), (512, 1)):
        (_, chi2_b, _, _, _, _), pb = _solve(probs, threads=nt, ctas_per_sm=cps)
        assert np.array_equal(chi2_a, chi2_b), (nt, cps)
        for x, y in zip(pa, pb):
            assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
    # one problem alone gives what it gave inside the batch
    for k in (0, len(probs) - 1):
        (_, chi2_1, _, _, _, _), p1 = _solve([probs[k]])
        assert chi2_1[0] == chi2_a[k]
        assert np.array_equal(p1[0][1], pa[k][1])


def test_autotune_keeps_results(probs):
    hs = [N.BAProblemGPU.from_ba(p, precision=N.PREC_FP64) for p in probs]
    b = N.PersistentBatch(hs)
    ref = b.lm_solve(N.LMSettings(**SET), threads=256, ctas_per_sm=1)
    for g, p in zip(hs, probs):
        g.set_params(p.cams, p.pts)
    nt, cps = b.autotune(N.LMSettings(**SET))
    assert nt in (128, 256, 512) and 1 <= cps <= 2
    for g, p in zip(hs, probs):
        g.set_params(p.cams, p.pts)
    out = b.lm_solve(N.LMSettings(**SET))
    assert np.array_equal(out[1], ref[1])
    b.close()
    for g in hs:
        g.close()


def test_batch_rejects_bad_input(probs):
    g = N.BAProblemGPU.from_ba(probs[0], precision=N.PREC_FP64)
    with pytest.raises(N.NelsonError):
        N.PersistentBatch([g, g])
    g.close()
