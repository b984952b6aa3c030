"""Bounded device waits run out instead of hanging, and the handle recovers.

The triangular solves' CTAs wait on each other's tile flags.  Every wait is
bounded by a poll count (nl_set_wait_limit).  nl_check_wait_timeout runs the
forward solve with the first tile's flag never published (its CTA is not
launched), so every other CTA's first wait must give up: the call returns
NL_ERR_TIMEOUT promptly, no kernel writes anything, and the next
computeIncrement on the same handle solves normally.  No GPU fault, trap or
endless loop is involved: the missing flag is a tile that was never
scheduled, and the wait that looks for it ends after the set number of polls.
"""
import time

import numpy as np
import pytest

from nelson_b200 import native as N
from nelson_b200.problems import make_config

pytestmark = pytest.mark.gpu

NL_ERR_TIMEOUT = 7


@pytest.mark.parametrize("prec", [N.PREC_FP64, N.PREC_MIXED])
def test_flag_wait_times_out_and_handle_recovers(prec):
    p = make_config(1, 0.1)  # 20 cameras x 9: a reduced system of two 128-row tiles
    assert -(-p.nc_var * p.bc // 128) >= 2
    g = N.BAProblemGPU.from_ba(p, precision=prec)
    g.update(True)
    mu = 1e-3 * g.max_abs_hdiag()
    assert g.compute_increment(0.0, mu)
    du0, dv0 = g.increment()
    # a short bound: the waits give up after 2,000 polls
    g.set_wait_limit(2000)
    t0 = time.perf_counter()
    assert g.check_wait_timeout() == NL_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 5.0
    # the default bound again: the same handle solves as before
    g.set_wait_limit(0)
    assert g.compute_increment(0.0, mu)
    du1, dv1 = g.increment()
    assert np.array_equal(du0, du1) and np.array_equal(dv0, dv1)
    g.close()


def test_check_needs_two_tiles():
    p = make_config(0, 0.3)  # 20 cameras x 6: one 128-row tile
    g = N.BAProblemGPU.from_ba(p, precision=N.PREC_FP64)
    assert -(-p.nc_var * p.bc // 128) == 1
    assert g.check_wait_timeout() == 2  # NL_ERR_STATE
    g.close()
