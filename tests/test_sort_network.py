"""The one-CTA sort's network (sort_one_block_kernel in mb2_sort.cu), run on the
host: a bitonic network over p2 = n rounded up to a power of two, stage (k, j)
comparing slot lo = 2t - (t mod j) with lo + j for t < p2 / 2, ascending where
lo & k == 0, over the composites key << 32 | position (padding all ones). Its
order must be a stable argsort's for every size the kernel takes, so that the
sort gives the permutation of the radix passes it stands in for. The device
kernel itself is checked against a host stable sort in the GPU tests."""
import numpy as np
import pytest


def network_order(keys):
    n = len(keys)
    p2 = 2
    while p2 < n:
        p2 *= 2
    comp = np.full(p2, np.iinfo(np.uint64).max, np.uint64)
    comp[:n] = (keys.astype(np.uint64) << np.uint64(32)) | np.arange(n, dtype=np.uint64)
    t = np.arange(p2 // 2)
    k = 2
    while k <= p2:
        j = k // 2
        while j > 0:
            lo = 2 * t - (t & (j - 1))
            hi = lo + j
            assert hi.max() < p2 and np.all((lo & j) == 0)
            a, b = comp[lo].copy(), comp[hi].copy()
            swap = (a > b) == ((lo & k) == 0)
            comp[lo] = np.where(swap, b, a)
            comp[hi] = np.where(swap, a, b)
            j //= 2
        k *= 2
    return (comp[:n] & np.uint64(0xFFFFFFFF)).astype(np.int64)


@pytest.mark.parametrize("n", [2, 3, 5, 31, 32, 33, 1000, 2047, 2048, 4096, 5000, 8191, 8192])
@pytest.mark.parametrize("distinct", [3, 1 << 30])
def test_network_is_a_stable_sort(n, distinct):
    rng = np.random.default_rng(n * 7 + distinct % 97)
    keys = rng.integers(0, distinct, n).astype(np.uint32)
    assert np.array_equal(network_order(keys), np.argsort(keys, kind="stable"))
