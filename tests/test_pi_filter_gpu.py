"""GPU parity of the permutation filter against the CPU restatement of pi_filter.cu, in rank
order, n = 1..11 (the packed-register kernels serve every n <= 16)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def cases():
    rng = np.random.Generator(np.random.PCG64(1375))
    out = [(1, [0], [0]), (2, [0, 1], [1, 0]), (3, [0, 1, 2], [0, 1, 2]), (3, [2, 1, 0], [0, 1, 2])]
    for n in (4, 5, 7, 8, 9, 10, 11):
        for _ in range(3):
            cl = int(rng.integers(3, n + 1))
            cycle = [int(v) for v in rng.permutation(n)[:cl]]
            triple = [int(v) for v in rng.permutation(n)[:3]]
            out.append((n, cycle, triple))
    return out


@pytest.mark.parametrize("skip", [False, True])
def test_pi_filter_matches_oracle(native_lib, oracle, skip):
    from tdp1375_b200 import GPUSortingSearch
    for n, cycle, triple in cases():
        hits, rows = oracle.pi_filter(cycle, triple, n, skip)
        got = GPUSortingSearch.filterPiPermutations(cycle, len(cycle), triple, len(triple), n, skip)
        # at most 1,048,576 rows come back (MAX_OUTPUT, pi_filter.cu:16), the first ones in rank order
        assert len(got) == min(hits, 1 << 20) and got == rows, (n, cycle, triple)


def test_pi_filter_row_limit_and_count(native_lib, oracle):
    import ctypes
    from tdp1375_b200 import native
    n, cycle, triple = 10, [0, 4, 1, 7, 3, 9, 2], [1, 5, 8]
    hits, rows = oracle.pi_filter(cycle, triple, n, False)
    assert hits > 100
    out = (ctypes.c_uint8 * (100 * n))()
    c8 = (ctypes.c_uint8 * len(cycle))(*cycle)
    t8 = (ctypes.c_uint8 * 3)(*triple)
    got = native_lib.tdp_pi_filter(c8, len(cycle), t8, 3, n, 0, out, 100)
    assert got == hits
    raw = bytes(out)
    assert [raw[r * n:(r + 1) * n] for r in range(100)] == rows[:100]
