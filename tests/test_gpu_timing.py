"""Phase timings of computeIncrement (nl_phase_timings, nl_set_timing_detail).

The default timing records the phases and the trailing-update launches only;
with the detail switch every step of the factorisation's critical path is
timed as well (one diagonal-tile factor per tile of S).  Timing changes how
the chain's kernels are launched, never what they compute: the increment is
bit-identical with and without it.
"""
import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import make_config

pytestmark = pytest.mark.gpu


def test_timing_detail_fills_the_critical_path_and_changes_no_result():
    p = make_config(1, 0.5)  # 100 cameras x 9 parameters: 8 tiles of 128
    g = N.BAProblemGPU.from_ba(p, precision=N.PREC_MIXED)
    g.update(True)
    mu = 1e-3 * g.max_abs_hdiag()

    assert g.compute_increment(0.0, mu)
    plain = [a.copy() for a in g.increment()]
    t = g.phase_times()
    assert t["total_ms"] > 0 and t["factor_ms"] > 0 and t["solve_ms"] > 0
    assert t["panels"] == 0 and t["panel_ms"] == 0 and t["first_ms"] == 0

    g.set_timing_detail(True)
    assert g.compute_increment(0.0, mu)
    detailed = [a.copy() for a in g.increment()]
    t = g.phase_times()
    ntiles = -(-p.nc_var * p.bc // 128)
    assert t["panels"] == ntiles
    assert t["panel_ms"] > 0 and t["first_ms"] > 0 and t["wait_ms"] >= 0

    g.set_timing_detail(False)
    assert g.compute_increment(0.0, mu)
    again = [a.copy() for a in g.increment()]
    assert g.phase_times()["panels"] == 0
    for a, b, c in zip(plain, detailed, again):
        assert np.array_equal(a, b) and np.array_equal(a, c)
    g.close()
