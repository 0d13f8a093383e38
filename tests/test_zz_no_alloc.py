"""The allocation-free permutation filter, called through the C ABI.

tdp_pi_filter_noalloc serves hosts that must not call cudaMalloc: a process whose own pool
allocator owns the device heap (a JVM or database runtime), or a real-time service that
allocates only at start-up.  It keeps its scratch in a static device array and writes rows
into a device buffer the caller owns.  This file is collected last on purpose, so a run that
stops at the first failure has run every other test first.  Each case is filtered twice in a
row (the second call reuses the scratch the first one left behind) and must give the hit
count and the rows, byte for byte, of both the allocating tdp_pi_filter and the oracle's
restatement of pi_filter.cu; a row limit below the hit count and n = 1 are covered, and a
size beyond the static scratch must be refused.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

# (n, cycle, oriented triple, skip the 2-move check, max_rows)
CASES = [
    (10, [0, 4, 1, 7, 3, 9, 2], [1, 5, 8], False, 1 << 18),
    (11, [2, 5, 9, 0, 7, 3], [4, 10, 6], True, 1 << 18),
    (10, [0, 4, 1, 7, 3, 9, 2], [1, 5, 8], False, 37),  # fewer rows than hits
    (1, [0], [0], False, 4),
]


def _u8(seq):
    return (ctypes.c_uint8 * max(1, len(seq)))(*seq)


def test_noalloc_filter_matches_allocating_filter_and_oracle_on_two_calls(oracle):
    import torch
    from tdp1375_b200 import native
    lib = native.load()
    stream = torch.cuda.Stream()
    for n, cycle, triple, skip, max_rows in CASES:
        hits, oracle_rows = oracle.pi_filter(cycle, triple, n, skip)
        want_rows = (ctypes.c_uint8 * (max_rows * n))()
        want = lib.tdp_pi_filter(_u8(cycle), len(cycle), _u8(triple), len(triple), n, int(skip), want_rows, max_rows)
        assert want == hits, native.last_error()
        rows = min(hits, max_rows)
        assert bytes(want_rows)[: rows * n] == b"".join(oracle_rows[:rows])
        for _call in range(2):
            with torch.cuda.stream(stream):  # the fill and the filter run in order on one stream
                out = torch.full((max_rows * n,), 255, dtype=torch.uint8, device="cuda")
                got = lib.tdp_pi_filter_noalloc(_u8(cycle), len(cycle), _u8(triple), len(triple), n, int(skip),
                                                ctypes.c_void_p(out.data_ptr()), max_rows,
                                                ctypes.c_void_p(stream.cuda_stream))
            stream.synchronize()
            assert got == hits, native.last_error()
            data = out.cpu().numpy().tobytes()
            assert data[: rows * n] == bytes(want_rows)[: rows * n]
            assert data[rows * n:] == b"\xff" * ((max_rows - rows) * n)  # nothing written past the limit


def test_noalloc_filter_rejects_sizes_beyond_its_scratch():
    import torch
    from tdp1375_b200 import native
    lib = native.load()
    out = torch.zeros(13, dtype=torch.uint8, device="cuda")
    rc = lib.tdp_pi_filter_noalloc(_u8([0, 1, 2]), 3, _u8([0, 1, 2]), 3, 13, 0, ctypes.c_void_p(out.data_ptr()), 1,
                                   ctypes.c_void_p(0))
    assert rc == native.ERR_ARGUMENT
    assert "n must be in 1..12" in native.last_error()
