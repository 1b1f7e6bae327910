"""The divide-free index maps of the sweep kernels (mgp_core.cuh: fastdiv24):
k / d as (k * ceil(2^24 / d)) >> 24, claimed exact for k < 16384 with
d <= 1024 and for k < 65536 with d <= 256 -- checked here for every pair."""
import numpy as np


def _exact(kmax, dmax):
    k = np.arange(kmax, dtype=np.uint64)
    for d in range(1, dmax + 1):
        m = np.uint64(((1 << 24) + d - 1) // d)
        assert m < (1 << 32)
        q = (k * m) >> np.uint64(24)
        if not np.array_equal(q, k // np.uint64(d)):
            return d
    return None


def test_fastdiv24_exact_small_divisors():
    assert _exact(65536, 256) is None


def test_fastdiv24_exact_level_sizes():
    assert _exact(16384, 1024) is None


def test_fastdiv24_fails_outside_its_range():
    """The bound is not slack: past k * (d - 1) ~ 2^24 the map goes wrong."""
    d = 1000
    k = np.arange(1 << 16, 1 << 17, dtype=np.uint64)
    m = np.uint64(((1 << 24) + d - 1) // d)
    assert not np.array_equal((k * m) >> np.uint64(24), k // np.uint64(d))
