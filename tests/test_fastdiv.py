"""The band reduction's division by one high multiply (csrc/super.cu, FastDiv): for 1 <= d and
0 <= n with n * d < 2^32, floor(n / d) == (n * m) >> 32 with m = floor((2^32 - 1) / d) + 1
(d = 1 divides by nothing). The kernel divides its loop indices, n < 16 rows x 8192 words, by row
lengths d <= 8192. Checked here at every d of that range on the values where a wrong quotient
would first show: each multiple of d and the value just below it. CPU only, exact integers."""
import numpy as np


def fast_div(n, d):
    if d == 1:
        return n
    m = np.uint64(0xFFFFFFFF // d + 1)
    return ((n.astype(np.uint64) * m) >> np.uint64(32)).astype(np.int64)


def test_fast_div_matches_floor_division_over_the_kernels_range():
    top = 16 * 8192
    for d in range(1, 8193):
        k = np.arange(0, top // d + 2, dtype=np.int64) * d
        n = np.concatenate([k, k - 1, k + d - 1])
        n = n[(n >= 0) & (n < top)]
        assert np.array_equal(fast_div(n, d), n // d), f"divisor {d}"


def test_fast_div_needs_the_range_bound():
    # outside n * d < 2^32 the identity can fail: the bound in the kernel's comment is needed
    d = 3
    m = 0xFFFFFFFF // d + 1
    n = next(v for v in range(0xAAAAAAAB - 4, 0xFFFFFFFF) if (v * m) >> 32 != v // d)
    assert n * d >= 1 << 32
