"""The tensor-core (tcgen05) trailing update against the CUDA-core update."""
import pytest

from nelson_b200 import native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ntiles,seed", [(2, 1), (3, 7), (9, 123)])
def test_tc_update_matches_cuda_core(ntiles, seed):
    # split-BF16x3 products: ~2^-16 relative per product, FP32 accumulation
    assert N.selftest_tc_update(ntiles, seed) < 2e-4
