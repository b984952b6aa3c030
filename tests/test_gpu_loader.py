"""Problems read from files solve on the GPU like generated ones: a BAL-style
file (written from a synthetic scene) and a synthetic problem on a
visibility list, LM traces against the FP64 oracle (1e-9 FP64, 1e-6 mixed)."""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200 import problems as P

pytestmark = pytest.mark.gpu

TOL = {N.PREC_FP64: 1e-9, N.PREC_MIXED: 1e-6}


def _trace_check(oracle_lib, p, prec):
    o = oracle_lib.Oracle.from_ba(p)
    g = N.BAProblemGPU.from_ba(p, precision=prec)
    _, tr_o, _, _ = o.lm_solve(oracle_lib.LMSettings(maxNumIt=6))
    _, tr_g, _, _ = g.lm_solve(N.LMSettings(maxNumIt=6))
    assert abs(tr_g[-1, 2] - tr_o[-1, 2]) <= TOL[prec] * tr_o[-1, 2]
    assert tr_g[-1, 2] < 0.5 * tr_g[0, 2]
    g.close()


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_bal_file_solves(tmp_path, oracle_lib, prec):
    p = P.make_config(1, 0.02)
    p.obs = p.obs - np.array([p.cx, p.cy])
    p.cx = p.cy = 0.0
    f = tmp_path / "scene.bal"
    P.save_bal(str(f), p)
    _trace_check(oracle_lib, P.load_bal(str(f)), prec)


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_visibility_list_solves(tmp_path, oracle_lib, prec):
    rng = np.random.default_rng(2)
    nc, npts = 24, 600
    cam = np.concatenate([rng.choice(nc, size=4, replace=False) for _ in range(npts)]).astype(np.int32)
    pt = np.repeat(np.arange(npts), 4).astype(np.int32)
    f = tmp_path / "vis.txt"
    P.save_pairs(str(f), nc, npts, cam, pt)
    nc2, np2, c2, p2 = P.load_pairs(str(f))
    _trace_check(oracle_lib, P.problem_from_pairs(nc2, np2, c2, p2, bc=9, seed=4), prec)
