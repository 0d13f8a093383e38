"""CPU check of the oracle's extension filter against an independent Python restatement of
the reference predicates (pi_filter.cu:55-115, CommonOperations.java:167-182, 406-445)."""
import ctypes
import itertools

import numpy as np


def cyclic(index, symbols):
    leaps = 0
    for i in range(len(symbols)):
        if index[symbols[i]] > index[symbols[(i + 1) % len(symbols)]]:
            leaps += 1
    return leaps <= 1


def has_2_move(index, cycle):
    pos = {s: i for i, s in enumerate(cycle)}
    L = len(cycle)
    before = L % 2
    for a, b, c in itertools.combinations(cycle, 3):
        if not cyclic(index, [a, b, c]):
            continue
        k = lambda x, y: (pos[y] - pos[x]) % L
        if (k(a, b) % 2) + (k(b, c) % 2) + (k(c, a) % 2) - before == 2:
            return True
    return False


def keep(spi, pi, added):
    n = len(pi)
    index = [0] * n
    for q, s in enumerate(pi):
        index[s] = q
    if not cyclic(index, list(added)):
        return False
    rindex = [n - 1 - index[s] for s in range(n)]
    seen, oriented = set(), False
    for s in range(n):
        if s in seen:
            continue
        cyc, cur = [], s
        while cur not in seen:
            seen.add(cur)
            cyc.append(cur)
            cur = spi[cur]
        if cyclic(rindex, cyc):
            continue
        oriented = True
        if has_2_move(index, cyc):
            return False
    return oriented


def extensions(spi, pi):
    n = len(pi)
    for a, b, c in itertools.combinations(range(n), 3):
        for o in (0, 1):
            r1, r2 = (b, c) if o == 0 else (c, b)
            rho = list(range(n))
            rho[a], rho[r1], rho[r2] = r1, r2, a
            yield [spi[rho[x]] for x in range(n)], list(pi), (a, r1, r2)
    for i, j, k in itertools.combinations(range(n + 3), 3):
        g = (i, j - 1, k - 2)
        for o in (0, 1):
            p2 = []
            for pos in range(n + 1):
                for w in range(3):
                    if g[w] == pos:
                        p2.append(n + w)
                if pos < n:
                    p2.append(pi[pos])
            s2 = list(spi) + [0, 0, 0]
            x, y, z = n, n + 1, n + 2
            if o == 0:
                s2[x], s2[y], s2[z] = y, z, x
                added = (x, y, z)
            else:
                s2[x], s2[z], s2[y] = z, y, x
                added = (x, z, y)
            yield s2, p2, added


def test_oracle_extension_filter_matches_python(oracle):
    L = oracle.lib()
    L.oracle_extension_filter.restype = ctypes.c_int64
    rng = np.random.Generator(np.random.PCG64(7))
    for trial in range(4):
        n = 9
        q = rng.permutation(n)
        spi = list(range(n))
        for t in range(3):
            a, b, c = sorted(int(v) for v in q[3 * t:3 * t + 3])
            if trial % 2 == 0:
                spi[a], spi[c], spi[b] = c, b, a  # unoriented 3-cycle (a c b)
            else:
                x, y, z = (int(v) for v in q[3 * t:3 * t + 3])
                spi[x], spi[y], spi[z] = y, z, x
        pi = list(range(n))
        want = [1 if keep(s2, p2, added) else 0 for s2, p2, added in extensions(spi, pi)]
        count = L.oracle_extension_count(n)
        assert count == len(want)
        out = (ctypes.c_uint8 * count)()
        hits = L.oracle_extension_filter(oracle._u8(spi), oracle._u8(pi), n, out)
        assert hits == sum(want)
        assert list(out) == want
