"""Extensions of a configuration by one cycle (Extensions.java:95-196, the proof generator's
extend step) and the signature operations they use.

A configuration is spi (successor array over 0..n-1, every symbol in a cycle of length >= 2)
with pi = (0 1 ... n-1).  Signatures are float arrays over pi positions
(Configuration.signature): the cycle's label by first appearance along pi, plus index/100 on
oriented cycles.  All float arithmetic follows Java's (float32, with the double steps where
the reference has them).

* ``type1_extensions``: for every open gate a and every b <= c (not a = b = c), a new
  unoriented 3-cycle inserted before positions a, b, c (Extensions.java:95-116);
* ``type2_extensions``: for a full configuration, every a <= b <= c (not all equal)
  (Extensions.java:118-141);
* ``type3_extensions``: an unoriented cycle grown by two symbols inserted before positions
  a <= b; kept when it stays unoriented with at most two open gates, or, for a 3-cycle that
  turns into an oriented 5-cycle, when that 5-cycle admits no 2-move (Extensions.java:143-196).

* ``combination_extensions``: a bad small component (oriented 5-cycle, interleaving pair,
  necklaces) inserted at every position (Combinations.java:31-46, 182-199).

Each extension is returned as (description, spi) with spi = Configuration.ofSignature of
the extended signature.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Set, Tuple

import numpy as np

F = np.float32


def cycles_in_order(spi: Sequence[int]) -> List[List[int]]:
    """Cycles of spi, each listed from its smallest symbol along spi."""
    seen, out = set(), []
    for s in range(len(spi)):
        if s in seen:
            continue
        c, cur = [], s
        while cur not in seen:
            seen.add(cur)
            c.append(cur)
            cur = spi[cur]
        out.append(c)
    return out


def cyclic_order(index: Sequence[int], symbols: Sequence[int]) -> bool:
    """CommonOperations.areSymbolsInCyclicOrder (CommonOperations.java:167-182): at most one
    leap of `index` going around `symbols`."""
    leaps = 0
    for i in range(len(symbols)):
        if index[symbols[i]] > index[symbols[(i + 1) % len(symbols)]]:
            leaps += 1
            if leaps > 1:
                return False
    return True


def signature(spi: Sequence[int]) -> List[np.float32]:
    """Configuration.signature under pi = (0 1 ... n-1) (Configuration.java:56-104)."""
    n = len(spi)
    inv_index = [n - 1 - p for p in range(n)]  # index of each symbol in pi^-1
    cyc = {}
    for c in cycles_in_order(spi):
        for s in c:
            cyc[s] = tuple(c)
    labels, oriented, out = {}, {}, []
    for p in range(n):
        c = cyc[p]
        if c not in oriented:
            oriented[c] = not cyclic_order(inv_index, c)
        if c not in labels:
            labels[c] = len(labels) + 1
        if oriented[c]:
            start = min(range(len(c)), key=lambda j: c[j])  # symbol at the smallest position
            idx = (c.index(p) - start) % len(c) + 1
            out.append(F(F(labels[c]) + F(F(idx) / F(100))))
        else:
            out.append(F(labels[c]))
    return out


def _frac(v: np.float32) -> bool:
    return float(v) % 1 > 0


def of_signature(sig: Sequence[float]) -> List[int]:
    """Configuration.ofSignature (Configuration.java:106-145) as a successor array."""
    n = len(sig)
    by_label, oriented = {}, {}
    for i in range(n - 1, -1, -1):
        v = F(sig[i])
        label = int(v)
        by_label.setdefault(label, []).append(i)
        if _frac(v):
            rank = int(math.floor(float(F(F(v - F(label)) * F(100))) + 0.5))
            oriented.setdefault(label, {})[rank] = i
    spi = list(range(n))
    for label, members in by_label.items():
        if label in oriented:
            ranks = oriented[label]
            members = [ranks[r] for r in sorted(ranks)]
        for k, s in enumerate(members):
            spi[s] = members[(k + 1) % len(members)]
    return spi


def open_gates(spi: Sequence[int]) -> Set[int]:
    """CommonOperations.getOpenGates (CommonOperations.java:501-546): symbols a with
    b = spi(a) such that no edge (c, spi(c)) of another cycle intersects (a, b) in pi^-1 and
    no c of a's cycle makes (a, b, c) cyclic in pi."""
    n = len(spi)
    pos = list(range(n))
    inv_index = [n - 1 - p for p in range(n)]
    cycles = [c for c in cycles_in_order(spi) if len(c) > 1]
    gates = set()
    for eps in cycles:
        for a in eps:
            b = spi[a]
            closed = False
            for gamma in cycles:
                if gamma is not eps:
                    if any(cyclic_order(inv_index, [a, c, b, spi[c]]) for c in gamma):
                        closed = True
                        break
                else:
                    if any(c != a and c != b and cyclic_order(pos, [a, b, c]) for c in eps):
                        closed = True
                        break
            if not closed:
                gates.add(a)
    return gates


def _insert_label(sig: Sequence[np.float32], label: int, positions: Sequence[int]) -> List[np.float32]:
    """Extensions.unorientedExtension: `label` inserted before each (sorted) position."""
    out = list(sig)
    for i, p in enumerate(sorted(positions)):
        out.insert(p + i, F(label))
    return out


def type1_extensions(spi: Sequence[int]) -> List[Tuple[str, List[int]]]:
    sig = signature(spi)
    new_label = len(cycles_in_order(spi)) + 1
    gates = open_gates(spi)
    out = []
    for i in range(len(sig)):
        if i in gates:
            for b in range(len(sig)):
                for c in range(b, len(sig)):
                    if not (i == b == c):
                        out.append((f"a={i} b={b} c={c}", of_signature(_insert_label(sig, new_label, [i, b, c]))))
    return out


def type2_extensions(spi: Sequence[int]) -> List[Tuple[str, List[int]]]:
    if open_gates(spi):
        return []
    sig = signature(spi)
    new_label = len(cycles_in_order(spi)) + 1
    out = []
    for a in range(len(sig)):
        for b in range(a, len(sig)):
            for c in range(b, len(sig)):
                if not (a == b == c):
                    out.append((f"a={a} b={b} c={c}", of_signature(_insert_label(sig, new_label, [a, b, c]))))
    return out


def _remains_unoriented(indexes: Sequence[int], *new: int) -> bool:
    """Extensions.remainsUnoriented: both new positions fall in one gap of the cycle."""
    gaps = set()
    for index in new:
        for i in range(len(indexes)):
            left, right = indexes[i], indexes[(i + 1) % len(indexes)]
            if (left < index <= right) or (right < left and (left < index or index <= right)):
                gaps.add((left, right))
    return len(gaps) == 1


def _float_cyclic(elements: Sequence[np.float32], other: Sequence[np.float32]) -> bool:
    """Extensions.areSymbolsInCyclicOrder(float[], float[]) (Extensions.java:198-219),
    statement for statement."""
    nxt = 0
    L = len(elements)
    for i in range(L):
        if elements[i] == other[nxt]:
            for j in range(L + 1):
                index = (i + j) % L
                if math.floor(float(elements[index])) == math.floor(float(other[nxt % len(other)])):
                    if elements[index] == other[nxt % len(other)]:
                        nxt += 1
                        if nxt > len(other):
                            return True
                    else:
                        return False
    return True


def _extend(cycle: Sequence[int], label: int, sig: Sequence[np.float32], a: int, b: int) -> List[np.float32]:
    """Extensions.extend (Extensions.java:221-244): the 3-cycle's symbols, from its largest,
    get label + 0.01 (i+1) (float += double), then label + 0.05 and label + 0.04 are
    inserted before positions a and b."""
    k = cycle.index(max(cycle))
    cyc = list(cycle[k:]) + list(cycle[:k])
    out = list(sig)
    for i in range(len(cyc) - 1, -1, -1):
        out[cyc[i]] = F(float(out[cyc[i]]) + 0.01 * (i + 1))
    nxt = F(0.05)
    inserted = 0
    for p in (a, b):
        out.insert(p + inserted, F(F(label) + nxt))
        nxt = F(nxt - F(0.01))
        inserted += 1
    return out


def type3_extensions(spi: Sequence[int]) -> List[Tuple[str, List[int]]]:
    sig = signature(spi)
    n = len(sig)
    sizes, indexes, cycle_of = {}, {}, {}
    cyc = {}
    for c in cycles_in_order(spi):
        for s in c:
            cyc[s] = c
    for i in range(n):
        label = int(math.floor(float(sig[i])))
        sizes[label] = sizes.get(label, 0) + 1
        indexes.setdefault(label, []).append(i)
        cycle_of.setdefault(label, cyc[i])
    out = []
    for label in range(1, len(cycles_in_order(spi)) + 1):
        if any(_frac(v) and math.floor(float(v)) == label for v in sig):
            continue
        for a in range(n):
            for b in range(a, n):
                ext = of_signature(_insert_label(sig, label, [a, b]))
                cycle_text = "(" + " ".join(str(x) for x in cycle_of[label]) + ")"
                if _remains_unoriented(indexes[label], a, b):
                    if len(open_gates(ext)) <= 2:
                        out.append((f"a={a} b={b}, extended cycle: {cycle_text}", ext))
                elif sizes[label] == 3:
                    prime = _extend(cycle_of[label], label, sig, a, b)
                    fractions = [F(F(x) + F(label)) for x in (0.01, 0.03, 0.05, 0.02, 0.04)]
                    if _float_cyclic(prime, fractions):  # otherwise it admits a 2-move
                        out.append((f"a={a} b={b}, extended cycle: {cycle_text}, turn oriented", of_signature(prime)))
    return out


# Combinations.java:31-46: the bad small components, in the reference's order.
BAD_SMALL_COMPONENTS = [
    "(0,3,1,4,2)",                                   # oriented 5-cycle
    "(0,4,2)(1,5,3)",                                # interleaving pair
    "(0,10,2)(1,5,3)(4,8,6)(7,11,9)",                # necklace of size 4
    "(0,7,5)(1,11,9)(2,6,4)(3,10,8)",                # twisted necklace of size 4
    "(0,4,2)(1,14,12)(3,7,5)(6,10,8)(9,13,11)",      # necklace of size 5
    "(0,16,2)(1,5,3)(4,8,6)(7,11,9)(10,14,12)(13,17,15)",  # necklace of size 6
]


def _successor_of(text: str) -> List[int]:
    import re
    cycles = [[int(t) for t in g.replace(",", " ").split()] for g in re.findall(r"\(([^()]*)\)", text)]
    n = max(max(c) for c in cycles) + 1
    succ = list(range(n))
    for c in cycles:
        for i, x in enumerate(c):
            succ[x] = c[(i + 1) % len(c)]
    return succ


def combination_extensions(spi: Sequence[int]) -> List[Tuple[str, List[int]]]:
    """SortOrExtendCombinations.extendCombinations (Combinations.java:182-199): for every bad
    small component and every position i < n, the component's signature with the
    configuration's cycle count added to each value (float) inserted at i."""
    sig = signature(spi)
    cycles = len(cycles_in_order(spi))
    out = []
    for b, text in enumerate(BAD_SMALL_COMPONENTS):
        comp = [F(v + F(cycles)) for v in signature(_successor_of(text))]
        for i in range(len(sig)):
            out.append((f"component={b} i={i}", of_signature(list(sig[:i]) + comp + list(sig[i:]))))
    return out
