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


def test_batch_matches_oracle(oracle_lib):
    probs = make_batch(6)
    hs = [N.BAProblemGPU.from_ba(p, precision=N.PREC_FP64) for p in probs]
    reasons, chi2, its, lat = N.lm_solve_batch(hs, N.LMSettings(maxNumIt=6))
    for k, p in enumerate(probs):
        o = oracle_lib.Oracle.from_ba(p)
        o.lm_solve(oracle_lib.LMSettings(maxNumIt=6))
        assert chi2[k] == pytest.approx(o.chi2(), rel=1e-9)
    for g in hs:
        g.close()


def test_batch_rejects_duplicates():
    p = make_batch(1)[0]
    g = N.BAProblemGPU.from_ba(p, precision=N.PREC_FP64)
    with pytest.raises(N.NelsonError):
        N.lm_solve_batch([g, g])
    g.close()
