"""Batched proof-generator frontier: SortOrExtend.compute / searchForSorting
(SortOrExtend.java:47-111) for a whole frontier of configurations at once.

For each configuration of the frontier the reference, one ForkJoin task at a time,
  1. takes its canonical form (Configuration.getCanonical) and lets SortingCoordinator admit
     one computation per canonical configuration (SortingCoordinator.java:72-100); a
     configuration already decided (its sorting or bad-case file exists) is not searched
     again;
  2. searches the canonical configuration in partial mode with ratio minRate = 2/maxRatio
     in stages: max depth 4, then min(upperBound, 8) if upperBound > 4, then
     min(upperBound, maxDepth) if upperBound > 8, where upperBound =
     floor(3-norm * (2 / minRate)) in float arithmetic; each stage is one JNI call.

`Frontier.resolve` does the same for a list of configurations with one canonicalisation
launch (tdp_canonical) and one batched search launch per stage (tdp_search_batch):
duplicates within the list and configurations decided by earlier calls are searched once.
The searched configuration is the canonical one; the returned sorting is on its symbols,
as SortOrExtend renders it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import api, casefile


def canonical_spi(spi: Sequence[int], variant: int) -> List[int]:
    """The configuration of an equivalent signature, relabelled so that its pi is
    (0 1 ... n-1): variant 2r reads spi with pi started at symbol r; variant 2r+1 is its
    mirror (spi conjugated by the involution that swaps the symbols at pi positions i and
    n-1-i, then inverted; Configuration.java:188-195).  This is the configuration that
    Configuration.ofSignature rebuilds from that signature."""
    n = len(spi)
    r, mirror = variant >> 1, variant & 1
    pos = [(x - r) % n for x in range(n)]
    sym = [(r + p) % n for p in range(n)]
    if not mirror:
        perm = list(spi)
    else:
        inv = [0] * n
        for x in range(n):
            inv[spi[x]] = x
        conj = [sym[n - 1 - pos[x]] for x in range(n)]
        perm = [conj[inv[conj[x]]] for x in range(n)]
    out = [0] * n
    for p in range(n):
        out[p] = pos[perm[sym[p]]]
    return out


def odd_cycles(spi: Sequence[int]) -> int:
    """The reference's "even cycles": cycles of odd length (MulticyclePermutation)."""
    return sum(len(c) % 2 for c in casefile.cycles_from_successor(spi))


def upper_bound(spi: Sequence[int], min_rate: np.float32) -> int:
    """floor(spi.get3Norm() * (2 / minRate)) with Java's int/float arithmetic
    (SortOrExtend.java:92)."""
    three_norm = (len(spi) - odd_cycles(spi)) // 2
    return int(math.floor(float(np.float32(three_norm) * (np.float32(2) / min_rate))))


@dataclass
class Resolution:
    key: bytes                      # canonical signature bytes (the coordinator's key)
    hash_code: int                  # Configuration.hashCode
    spi: List[int]                  # canonical configuration
    found: bool
    moves: List[Tuple[int, int, int]] = field(default_factory=list)  # symbol 3-cycles on spi
    depth_limit: int = 0            # max depth of the stage that decided it


class Frontier:
    def __init__(self, slot: int = 0, max_ratio: float = 1.375, max_depth: int = 11):
        self.slot = slot
        self.min_rate = np.float32(2) / np.float32(max_ratio)
        self.max_depth = max_depth
        self.decided: Dict[bytes, Resolution] = {}
        self.stage_counts: List[Tuple[int, int, int]] = []  # (stage, searched, found) per stage
        self.last_new: List[Resolution] = []  # configurations first decided by the last call

    def _stages(self, ub: int) -> List[int]:
        out = [4]
        if ub > 4:
            out.append(min(ub, 8))
        if ub > 8:
            out.append(min(ub, self.max_depth))
        return out

    def resolve(self, spis: Sequence[Sequence[int]]) -> List[Resolution]:
        sig, hashes, variants = canonical_batch(spis)
        keys = [sig[r, :len(s)].tobytes() for r, s in enumerate(spis)]
        todo: Dict[bytes, Resolution] = {}
        for r, s in enumerate(spis):
            k = keys[r]
            if k in self.decided or k in todo:
                continue
            todo[k] = Resolution(k, int(hashes[r]), canonical_spi(s, int(variants[r])), False)
        pending = list(todo.values())
        stage = 0
        while pending:
            batch = []
            for res in pending:
                stages = self._stages(upper_bound(res.spi, self.min_rate))
                if stage < len(stages):
                    res.depth_limit = stages[stage]
                    batch.append(res)
            if not batch:
                break
            groups: Dict[int, List[Resolution]] = {}
            for res in batch:
                groups.setdefault(res.depth_limit, []).append(res)
            found_here = 0
            for depth, group in groups.items():
                cases = [(list(range(len(g.spi))), g.spi, odd_cycles(g.spi)) for g in group]
                results = api.search_batch(self.slot, api.make_instances(cases, depth, False), len(cases),
                                           float(self.min_rate))
                for g, (pi, _, _), out in zip(group, cases, results):
                    if out.status == 1:
                        pos = [[out.positions[3 * d + t] for t in range(3)] for d in range(out.depth)]
                        g.moves = [tuple(m) for m in api.positions_to_symbols(pi, pos)]
                        g.found = True
                        found_here += 1
                    elif out.status != 0:
                        raise RuntimeError(f"search status {out.status}")
            self.stage_counts.append((stage, len(batch), found_here))
            pending = [res for res in batch if not res.found]
            stage += 1
        self.decided.update(todo)
        self.last_new = list(todo.values())
        return [self.decided[k] for k in keys]


def canonical_batch(spis: Sequence[Sequence[int]]):
    """(signatures, hash codes, variants) of the configurations, one tdp_canonical call."""
    import ctypes

    from . import native
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
    return sig, h, v
