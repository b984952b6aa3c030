"""Batched LM (nl_lm_solve_batch): many uneven problems of the batched
configuration's generator (6-parameter cameras U{8..64}, points U{200..4000},
k~U{3..8}) solved at once give the same results as solving them one by one
(the same kernels run in the same order per problem), and the one-by-one
results match the FP64 oracle (1e-9 FP64, 1e-6 mixed)."""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import make_batch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_batch_equals_single(prec):
    probs = make_batch(12)
    settings = N.LMSettings(maxNumIt=8)
    single = []
    for p in probs:
        g = N.BAProblemGPU.from_ba(p, precision=prec)
        _, tr, _, _ = g.lm_solve(settings, trace_cap=1)
        single.append((g.chi2(), g.get_params()[1]))
        g.close()
    hs = [N.BAProblemGPU.from_ba(p, precision=prec) for p in probs]
    reasons, chi2, its, lat = N.lm_solve_batch(hs, settings)
    for k, g in enumerate(hs):
        assert chi2[k] == pytest.approx(single[k][0], rel=1e-12), k
        assert np.abs(g.get_params()[1] - single[k][1]).max() <= 1e-9 * np.abs(single[k][1]).max()
        assert lat[k] > 0.0
    # a second batch on the same handles replays the captured sub-iterations
    for g, p in zip(hs, probs):
        g.set_params(p.cams, p.pts)
    reasons2, chi2b, _, lat2 = N.lm_solve_batch(hs, settings)
    assert np.array_equal(chi2b, chi2)
    for g in hs:
        g.close()


@pytest.mark.parametrize("prec,tol", [(N.PREC_FP64, 1e-9), (N.PREC_MIXED, 1e-6)])
def test_batch_matches_oracle(oracle_lib, prec, tol):
    """Every problem of a 24-problem batch against the oracle's LM on the same
    problem: final cost (1e-9 FP64, 1e-6 mixed), iteration count and
    termination reason, and the points."""
    probs = make_batch(24)
    hs = [N.BAProblemGPU.from_ba(p, precision=prec) for p in probs]
    reasons, chi2, its, lat = N.lm_solve_batch(hs, N.LMSettings(maxNumIt=6))
    for k, p in enumerate(probs):
        o = oracle_lib.Oracle.from_ba(p)
        r_o, _, it_o, _ = o.lm_solve(oracle_lib.LMSettings(maxNumIt=6))
        assert chi2[k] == pytest.approx(o.chi2(), rel=tol), k
        assert reasons[k] == r_o and its[k] == it_o, k
        pts_o = o.get_params()[1]
        # gauge-free problems: the points agree to the cost's precision
        assert np.abs(hs[k].get_params()[1] - pts_o).max() <= (1e-6 if prec == N.PREC_FP64 else 1e-3) * \
            np.abs(pts_o).max(), k
    for g in hs:
        g.close()


def test_batch_rejects_duplicates():
    p = make_batch(1)[0]
    g = N.BAProblemGPU.from_ba(p, precision=N.PREC_FP64)
    with pytest.raises(N.NelsonError):
        N.lm_solve_batch([g, g])
    g.close()
