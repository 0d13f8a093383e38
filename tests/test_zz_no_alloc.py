"""The allocation-free permutation filter against the allocating one.

tdp_pi_filter_noalloc is for callers that cannot allocate device memory: code running
while a CUDA stream is being captured, hosts whose own allocator owns the device heap, and
real-time hosts that forbid allocation once running.  It keeps its scratch in a static
device array and writes rows into a device buffer the caller owns.  This file is collected
last on purpose.  It makes two calls in a row through the C ABI and requires the same hit
counts and the same rows, byte for byte, as tdp_pi_filter; it also checks the size-limit
error.
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

CASES = [
    (10, [0, 4, 1, 7, 3, 9, 2], [1, 5, 8], False),
    (11, [2, 5, 9, 0, 7, 3], [4, 10, 6], True),
]


def _u8(seq):
    return (ctypes.c_uint8 * max(1, len(seq)))(*seq)


def test_noalloc_filter_matches_allocating_filter_on_two_calls():
    import torch
    from tdp1375_b200 import native
    lib = native.load()
    max_rows = 1 << 18
    stream = torch.cuda.Stream()
    for n, cycle, triple, skip in CASES:
        want_rows = (ctypes.c_uint8 * (max_rows * n))()
        want = lib.tdp_pi_filter(_u8(cycle), len(cycle), _u8(triple), len(triple), n, int(skip), want_rows, max_rows)
        assert want > 0, native.last_error()
        out = torch.full((max_rows * n,), 255, dtype=torch.uint8, device="cuda")
        got = lib.tdp_pi_filter_noalloc(_u8(cycle), len(cycle), _u8(triple), len(triple), n, int(skip),
                                        ctypes.c_void_p(out.data_ptr()), max_rows,
                                        ctypes.c_void_p(stream.cuda_stream))
        assert got == want, native.last_error()
        rows = min(want, max_rows)
        assert out[: rows * n].cpu().numpy().tobytes() == bytes(want_rows)[: rows * n]


def test_noalloc_filter_rejects_sizes_beyond_its_scratch():
    import torch
    from tdp1375_b200 import native
    lib = native.load()
    out = torch.zeros(13, dtype=torch.uint8, device="cuda")
    rc = lib.tdp_pi_filter_noalloc(_u8([0, 1, 2]), 3, _u8([0, 1, 2]), 3, 13, 0, ctypes.c_void_p(out.data_ptr()), 1,
                                   ctypes.c_void_p(0))
    assert rc == native.ERR_ARGUMENT
    assert "n must be in 1..12" in native.last_error()
