"""ctypes wrapper of the CPU oracle (oracle/tdp_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the checker and
by bench.py's CPU-baseline leg.  The product never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libtdp_oracle.so")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.oracle_count_even_cycles.argtypes = [_u8p, ctypes.c_int]
        L.oracle_rule_eval.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int]
        L.oracle_search_gpu_rule.argtypes = [_u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_uint64, _i32p, _i32p, _u64p]
        L.oracle_search_cpu_rule.argtypes = [_u8p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                             ctypes.c_uint64, _i32p, _i32p, _u64p]
        L.oracle_replay_positions.argtypes = [_u8p, _u8p, ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_float, ctypes.c_int, _i32p]
        L.oracle_replay_symbols.argtypes = [_u8p, _u8p, ctypes.c_int, _i32p, ctypes.c_int, _u8p]
        L.oracle_pi_filter.restype = ctypes.c_int64
        L.oracle_pi_filter.argtypes = [_u8p, ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _u8p,
                                       ctypes.c_int64]
        L.oracle_pi_filter_keep.argtypes = [_u8p, ctypes.c_int, _u8p, ctypes.c_int, _u8p, ctypes.c_int, ctypes.c_int]
        _f32p = ctypes.POINTER(ctypes.c_float)
        L.oracle_signature.argtypes = [_u8p, ctypes.c_int, _f32p]
        L.oracle_equivalent_signatures.argtypes = [_u8p, ctypes.c_int, _f32p]
        L.oracle_signature_hash.argtypes = [_f32p, ctypes.c_int]
        L.oracle_signature_hash.restype = ctypes.c_int32
        L.oracle_canonical.argtypes = [_u8p, ctypes.c_int, _f32p, _i32p, _i32p]
        _lib = L
    return _lib


def _u8(seq):
    seq = [int(v) & 0xFF for v in seq]
    return (ctypes.c_uint8 * max(1, len(seq)))(*seq)


def count_even(spi) -> int:
    return lib().oracle_count_even_cycles(_u8(spi), len(spi))


def rule_eval(n, initial_even, min_rate, max_depth, full, even, depth) -> int:
    """bit0 satisfies_rate, bit1 can_still_reach (sorting_search.cu:321-362)."""
    return lib().oracle_rule_eval(n, initial_even, ctypes.c_float(min_rate), max_depth, 1 if full else 0, even, depth)


def search_gpu_rule(pi, spi, initial_even, min_rate, max_depth, full, dedup=True, tight=False, node_limit=0,
                    commute=False):
    """Returns (status, positions[[i,j,k]...], (expanded, children)); status 1/0, -2 node limit.
    commute: skip children that commute with the incoming move in the other order (the
    engine's partial-order reduction, restated for cross-checking)."""
    pos = (ctypes.c_int * 48)()
    depth = ctypes.c_int(0)
    stats = (ctypes.c_uint64 * 2)()
    mode = (1 if dedup else 0) | (2 if tight else 0) | (4 if commute else 0)
    st = lib().oracle_search_gpu_rule(_u8(pi), _u8(spi), len(pi), initial_even, ctypes.c_float(min_rate), max_depth,
                                      1 if full else 0, mode, node_limit, pos, ctypes.byref(depth), stats)
    moves = [[pos[3 * d], pos[3 * d + 1], pos[3 * d + 2]] for d in range(depth.value)]
    return st, moves, (int(stats[0]), int(stats[1]))


def search_cpu_rule(pi, spi, initial_even, min_rate, max_moves, node_limit=0):
    """SortingSearch.java restatement. Returns (status, symbols[[a,b,c]...], expanded)."""
    sym = (ctypes.c_int * 48)()
    depth = ctypes.c_int(0)
    stats = (ctypes.c_uint64 * 2)()
    st = lib().oracle_search_cpu_rule(_u8(pi), _u8(spi), len(pi), initial_even, ctypes.c_float(min_rate), max_moves,
                                      node_limit, sym, ctypes.byref(depth), stats)
    moves = [[sym[3 * d], sym[3 * d + 1], sym[3 * d + 2]] for d in range(depth.value)]
    return st, moves, int(stats[0])


def replay_positions(pi, spi, positions, initial_even, min_rate, full):
    """(valid, symbols): GPUSortingSearch.java:65-74 replay + success test."""
    flat = [int(v) for m in positions for v in m]
    arr = (ctypes.c_int * max(3, len(flat)))(*flat)
    sym = (ctypes.c_int * max(3, len(flat)))()
    ok = lib().oracle_replay_positions(_u8(pi), _u8(spi), len(pi), arr, len(positions), initial_even,
                                       ctypes.c_float(min_rate), 1 if full else 0, sym)
    return bool(ok), [[sym[3 * d], sym[3 * d + 1], sym[3 * d + 2]] for d in range(len(positions))]


def replay_symbols(pi, spi, symbols):
    """Applies symbol 3-cycles; returns (final even count or -1 if a move is invalid, final spi)."""
    flat = [int(v) for m in symbols for v in m]
    arr = (ctypes.c_int * max(3, len(flat)))(*flat)
    out = (ctypes.c_uint8 * max(1, len(spi)))()
    even = lib().oracle_replay_symbols(_u8(pi), _u8(spi), len(pi), arr, len(symbols), out)
    return even, list(out)[: len(spi)]


def pi_filter(cycle, triple, n, skip_2move, max_out=1 << 20):
    """(hits, rows) in lexicographic rank order."""
    out = (ctypes.c_uint8 * max(1, max_out * n))()
    hits = lib().oracle_pi_filter(_u8(cycle), len(cycle), _u8(triple), len(triple), n, 1 if skip_2move else 0, out,
                                  max_out)
    rows = min(int(hits), max_out)
    raw = bytes(out)[: rows * n]
    return int(hits), [raw[r * n:(r + 1) * n] for r in range(rows)]


def pi_filter_keep(pi, cycle, triple, skip_2move) -> bool:
    return bool(lib().oracle_pi_filter_keep(_u8(pi), len(pi), _u8(cycle), len(cycle), _u8(triple), len(triple),
                                            1 if skip_2move else 0))


def parse_cycles(text: str):
    """Successor array of a permutation written in cycle notation, e.g. "(0 9 7)(1 5 2 6 3)";
    n is the largest symbol + 1 (the reference's configurations cover every symbol)."""
    import re
    cycles = [[int(t) for t in grp.replace(",", " ").split()] for grp in re.findall(r"\(([^()]*)\)", text)]
    n = max(max(c) for c in cycles) + 1
    succ = list(range(n))
    for c in cycles:
        for i, x in enumerate(c):
            succ[x] = c[(i + 1) % len(c)]
    return succ


def signature(spi):
    n = len(spi)
    out = (ctypes.c_float * n)()
    assert lib().oracle_signature(_u8(spi), n, out) == 0
    return list(out)


def equivalent_signatures(spi):
    n = len(spi)
    out = (ctypes.c_float * (2 * n * n))()
    assert lib().oracle_equivalent_signatures(_u8(spi), n, out) == 0
    return [list(out[v * n:(v + 1) * n]) for v in range(2 * n)]


def signature_hash(sig) -> int:
    arr = (ctypes.c_float * len(sig))(*sig)
    return int(lib().oracle_signature_hash(arr, len(sig)))


def canonical(spi):
    """(canonical signature, hash code, variant index) of Configuration.getCanonical."""
    n = len(spi)
    out = (ctypes.c_float * n)()
    h, v = ctypes.c_int32(), ctypes.c_int32()
    assert lib().oracle_canonical(_u8(spi), n, out, ctypes.byref(h), ctypes.byref(v)) == 0
    return list(out), h.value, v.value
