"""The tensor-core (tcgen05) trailing update against the CUDA-core update."""
import pytest

from nelson_b200 import native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ntiles,seed", [(2, 1), (3, 7), (9, 123)])
def test_tc_update_matches_cuda_core(ntiles, seed):
    # split-BF16x3 products: ~2^-16 relative per product, FP32 accumulation
    assert N.selftest_tc_update(ntiles, seed) < 2e-4


def test_blocked_diagonal_factor_matches_rank4_kernel():
    """The mixed path's 32-blocked diagonal-tile factor against the rank-4
    register kernel on a random SPD FP32 tile: L and inv(L) agree to FP32
    rounding (different operation orders), and the blocked kernel is timed."""
    for seed in (1, 2, 3):
        el, ei, us_b, us_r = N.selftest_potrf32(seed)
        print(f"seed {seed}: |dL| {el:.2e}  |dLinv| {ei:.2e}  blocked {us_b:.1f} us  rank-4 {us_r:.1f} us")
        assert el <= 2e-5 and ei <= 2e-4
