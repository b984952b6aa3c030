"""The tensor-core (tcgen05) trailing update against the CUDA-core update."""
import pytest

from nelson_b200 import native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ntiles,seed", [(2, 1), (3, 7), (9, 123)])
def test_tc_update_matches_cuda_core(ntiles, seed):
    # split-BF16x3 products: ~2^-16 relative per product, FP32 accumulation
    assert N.selftest_tc_update(ntiles, seed) < 2e-4


@pytest.mark.parametrize("ntiles,npanels,seed", [(3, 1, 5), (6, 2, 9), (9, 4, 3), (20, 3, 11)])
def test_tc_update_with_packed_panels(ntiles, npanels, seed):
    """The rank-(128 npanels) update of the factorisation's panel groups (one
    launch, npanels packed panels) against the CUDA-core update applied panel
    by panel."""
    err, ms = N.selftest_tc_update_k(ntiles, npanels, seed, reps=1)
    assert err < 2e-4 and ms > 0
