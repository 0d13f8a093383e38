"""ctypes wrapper of the reference's own CUDA search and permutation filter.

TEST INFRASTRUCTURE ONLY: oracle/_ref/libtdp_ref.so is the reference's sorting_search.cu,
slot_manager.cu and pi_filter.cu compiled from the reference sources for sm_100a with the
C driver oracle/ref_harness.cu (`make -C oracle ref`).  Tests, the fixture generators under
tests/golden/ and bench.py's reference legs use it to run the reference kernel on the same
inputs as this project's kernels; the product never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libtdp_ref.so")
LIB_DEBUG = os.path.join(HERE, "_ref", "libtdp_ref_g.so")  # device code unoptimised (make ref-debug)

NOT_FOUND, FOUND, TIMED_OUT, OVERFLOW, ERROR = 0, 1, 2, 3, -1
STATUS_NAME = {NOT_FOUND: "not_found", FOUND: "found", TIMED_OUT: "timeout", OVERFLOW: "overflow", ERROR: "error"}

_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_libs = {}


def build(reference_root: str) -> str:
    """Compiles oracle/_ref/libtdp_ref.so from the reference checkout at reference_root."""
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={reference_root}"], check=True)
    return LIB


def available(debug: bool = False) -> bool:
    return os.path.exists(LIB_DEBUG if debug else LIB)


def lib(debug: bool = False) -> ctypes.CDLL:
    """The optimised build, or with debug=True the build whose device code is unoptimised
    (make -C oracle ref-debug); both can be loaded in one process."""
    path = LIB_DEBUG if debug else LIB
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is not built (make -C oracle ref ref-debug REF=<reference checkout>)")
        L = ctypes.CDLL(path)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_init.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_longlong, ctypes.c_int]
        L.ref_search.argtypes = [ctypes.c_int, _u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_double, _i32p, _i32p, ctypes.POINTER(ctypes.c_double)]
        L.ref_pi_filter.restype = ctypes.c_longlong
        L.ref_pi_filter.argtypes = [_u8p, ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _u8p,
                                    ctypes.c_longlong]
        _libs[path] = L
    return _libs[path]


def last_error(debug: bool = False) -> str:
    return lib(debug).ref_last_error().decode()


def _u8(seq):
    seq = [int(v) & 0xFF for v in seq]
    return (ctypes.c_uint8 * max(1, len(seq)))(*seq)


def init(slots: int = 1, devices: int = 1, queue_bytes: int = 3000 << 20, dedup_entries: int = 1 << 21) -> None:
    """initGpuSortSlots: slot s on device s % devices, queue budget in bytes, table in entries."""
    if lib().ref_init(slots, devices, queue_bytes, dedup_entries) != 0:
        raise RuntimeError(last_error())


def destroy() -> None:
    if lib().ref_destroy() != 0:
        raise RuntimeError(last_error())


def search(pi, spi, initial_even, min_rate, max_depth, full, timeout_s=60.0, slot=0):
    """performGpuSortingSearch.  Returns (status, positions [[i,j,k], ...], wall ms)."""
    n = len(pi)
    pos = (ctypes.c_int32 * 48)()
    depth = ctypes.c_int32(0)
    ms = ctypes.c_double(0.0)
    st = lib().ref_search(slot, _u8(pi), _u8(spi), n, int(initial_even), ctypes.c_float(float(min_rate)),
                          int(max_depth), 1 if full else 0, float(timeout_s), pos, ctypes.byref(depth),
                          ctypes.byref(ms))
    if st == ERROR:
        raise RuntimeError(last_error())
    moves = [[pos[3 * d], pos[3 * d + 1], pos[3 * d + 2]] for d in range(depth.value)]
    return st, moves, ms.value


def pi_filter(cycle, triple, n, skip_2move, max_rows=1 << 20, debug=False):
    """performGpuPiFilter.  Returns the hit rows (bytes of length n) sorted, so that runs with
    the reference's arbitrary row order compare as sets."""
    out = (ctypes.c_uint8 * max(1, max_rows * n))()
    rows = lib(debug).ref_pi_filter(_u8(cycle), len(cycle), _u8(triple), len(triple), n, 1 if skip_2move else 0, out,
                                    max_rows)
    if rows < 0:
        raise RuntimeError(last_error(debug))
    raw = bytes(out)[: min(rows, max_rows) * n]
    return sorted(raw[r * n:(r + 1) * n] for r in range(min(rows, max_rows)))
