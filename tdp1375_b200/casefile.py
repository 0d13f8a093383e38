"""Case files: the "spi->[moves]" text the reference reads into its sorting tables
(AbstractSbtAlgorithm.loadSortings, AbstractSbtAlgorithm.java:166-179; Silvaetal.java:151-165)
and writes from its case generators (Cases3_2.java:19, EHCases.java:69).

A line is the configuration's spi in cycle notation followed by "->" and the sorting as a
list of 3-cycles on symbols, e.g.

    (0 4 2)(1 5 3)->[(0 2 4), (1 5 3), (0 2 4)]

The text is normalised the way the reference prints it: every cycle starts at its smallest
symbol (Cycle.defaultStringRepresentation, Cycle.java:100-114); spi's cycles follow their
smallest symbols, the order in which Configuration.ofSignature builds a canonical spi.

Records are (spi, moves): spi the successor array over 0..n-1, moves a list of symbol
triples (a, b, c) meaning the 3-cycle (a b c).  `sortings_table` keys records by
Configuration.hashCode computed on the GPU (tdp_canonical), like loadSortings does.
"""
from __future__ import annotations

import ctypes
import re
from typing import Dict, Iterable, List, Sequence, Tuple

import numpy as np

from . import native

Record = Tuple[List[int], List[Tuple[int, int, int]]]

_CYCLE = re.compile(r"\(([^()]*)\)")


def cycles_of(text: str) -> List[List[int]]:
    return [[int(t) for t in grp.replace(",", " ").split()] for grp in _CYCLE.findall(text)]


def successor(cycles: Sequence[Sequence[int]]) -> List[int]:
    """Successor array of a permutation given by cycles covering 0..n-1."""
    symbols = sorted(s for c in cycles for s in c)
    n = len(symbols)
    if symbols != list(range(n)):
        raise ValueError("cycles must cover 0..n-1 exactly once")
    succ = list(range(n))
    for c in cycles:
        for i, s in enumerate(c):
            succ[s] = c[(i + 1) % len(c)]
    return succ


def cycles_from_successor(spi: Sequence[int]) -> List[List[int]]:
    """Cycles of a successor array, each from its smallest symbol, ordered by that symbol."""
    seen = [False] * len(spi)
    out = []
    for s in range(len(spi)):
        if seen[s]:
            continue
        cyc, cur = [], s
        while not seen[cur]:
            seen[cur] = True
            cyc.append(cur)
            cur = spi[cur]
        out.append(cyc)
    return out


def _cycle_text(c: Sequence[int]) -> str:
    k = c.index(min(c))
    c = list(c[k:]) + list(c[:k])
    return "(" + " ".join(str(x) for x in c) + ")"


def parse_line(line: str) -> Record:
    """One case line -> (spi successor array, [(a, b, c), ...])."""
    left, right = line.strip().split("->")
    spi = successor(cycles_of(left))
    moves = [tuple(c) for c in cycles_of(right)]
    for m in moves:
        if len(m) != 3:
            raise ValueError(f"a move must be a 3-cycle: {m}")
    return spi, moves


def format_line(spi: Sequence[int], moves: Iterable[Sequence[int]]) -> str:
    left = "".join(_cycle_text(c) for c in cycles_from_successor(spi))
    return left + "->[" + ", ".join(_cycle_text(m) for m in moves) + "]"


def read_case_file(path: str) -> List[Record]:
    with open(path) as fh:
        return [parse_line(line) for line in fh if line.strip()]


def write_case_file(path: str, records: Iterable[Record]) -> None:
    with open(path, "w") as fh:
        for spi, moves in records:
            fh.write(format_line(spi, moves) + "\n")


def apply_moves(spi: Sequence[int], moves: Iterable[Sequence[int]]) -> List[int]:
    """spi after the moves, each (a b c) applied as spi o (a b c)^-1 (the search's update
    spi'[a] = spi[c], spi'[b] = spi[a], spi'[c] = spi[b])."""
    s = list(spi)
    for a, b, c in moves:
        s[a], s[b], s[c] = s[c], s[a], s[b]
    return s


def hash_codes(spis: Sequence[Sequence[int]]) -> np.ndarray:
    """Configuration.hashCode of each spi (pi = (0 1 ... n-1)), on the GPU."""
    count = len(spis)
    rows = np.zeros((count, 64), np.uint8)
    ns = np.zeros(count, np.uint8)
    for r, s in enumerate(spis):
        rows[r, :len(s)] = s
        ns[r] = len(s)
    sig = np.zeros((count, 64), np.float32)
    h = np.zeros(count, np.int32)
    v = np.zeros(count, np.int32)
    vp = ctypes.c_void_p
    rc = native.load().tdp_canonical(rows.ctypes.data_as(vp), ns.ctypes.data_as(vp), count, sig.ctypes.data_as(vp),
                                     h.ctypes.data_as(vp), v.ctypes.data_as(vp))
    if rc != 0:
        raise RuntimeError(native.last_error())
    return h


def sortings_table(records: Sequence[Record]) -> Dict[int, List[Record]]:
    """Records keyed by Configuration.hashCode, as loadSortings fills its multimap."""
    table: Dict[int, List[Record]] = {}
    for rec, h in zip(records, hash_codes([r[0] for r in records])):
        table.setdefault(int(h), []).append(rec)
    return table
