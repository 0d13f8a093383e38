"""GPU parity of the batched extension filter with the CPU restatement (oracle)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bases(count, unoriented, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    spi = np.zeros((count, 64), np.uint8)
    pi = np.zeros((count, 64), np.uint8)
    for b in range(count):
        q = rng.permutation(18)
        s = np.arange(18)
        for t in range(6):
            if unoriented:
                a, m, c = sorted(int(v) for v in q[3 * t:3 * t + 3])
                s[a], s[c], s[m] = c, m, a
            else:
                x, y, z = (int(v) for v in q[3 * t:3 * t + 3])
                s[x], s[y], s[z] = y, z, x
        spi[b, :18] = s
        pi[b, :18] = np.arange(18)
    return spi, pi


@pytest.mark.parametrize("unoriented", [True, False])
def test_extension_filter_matches_oracle(native_lib, oracle, unoriented):
    L = oracle.lib()
    L.oracle_extension_filter.restype = ctypes.c_int64
    count = 24
    spi, pi = bases(count, unoriented, 1375 + int(unoriented))
    per = native_lib.tdp_extension_count(18)
    assert per == 2 * 816 + 2 * 1330
    keep = np.zeros(count * per, np.uint8)
    hits = native_lib.tdp_extension_filter(spi.ctypes.data_as(ctypes.c_void_p), pi.ctypes.data_as(ctypes.c_void_p),
                                           18, count, keep.ctypes.data_as(ctypes.c_void_p))
    want_total = 0
    for b in range(count):
        want = (ctypes.c_uint8 * per)()
        want_total += L.oracle_extension_filter(oracle._u8(spi[b, :18]), oracle._u8(pi[b, :18]), 18, want)
        assert bytes(keep[b * per:(b + 1) * per]) == bytes(want), b
    assert hits == want_total
    if unoriented:
        assert hits > count


def test_extension_filter_seeded_bases_match_oracle(native_lib, oracle):
    """The seeded m=6 bases of the extension workload: hit list and count bit-exact."""
    from tdp1375_b200.cases import extension_bases
    L = oracle.lib()
    L.oracle_extension_filter.restype = ctypes.c_int64
    count = 64
    pi, spi, n = extension_bases(count)
    per = native_lib.tdp_extension_count(n)
    keep = np.zeros(count * per, np.uint8)
    hits = native_lib.tdp_extension_filter(spi.ctypes.data_as(ctypes.c_void_p), pi.ctypes.data_as(ctypes.c_void_p),
                                           n, count, keep.ctypes.data_as(ctypes.c_void_p))
    want_total = 0
    for b in range(count):
        want = (ctypes.c_uint8 * per)()
        want_total += L.oracle_extension_filter(oracle._u8(spi[b, :n]), oracle._u8(pi[b, :n]), n, want)
        assert bytes(keep[b * per:(b + 1) * per]) == bytes(want), b
    assert hits == want_total
