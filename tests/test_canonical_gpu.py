"""GPU parity of the batched canonical form with the oracle and the reference's golden
values (Configuration.getCanonical / hashCode)."""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "configuration_golden.json")))["configurations"]


def rows_of(perms):
    spi = np.zeros((len(perms), 64), np.uint8)
    ns = np.zeros(len(perms), np.uint8)
    for r, p in enumerate(perms):
        spi[r, :len(p)] = p
        ns[r] = len(p)
    return spi, ns


def run(native_lib, perms):
    spi, ns = rows_of(perms)
    sig = np.zeros((len(perms), 64), np.float32)
    h = np.zeros(len(perms), np.int32)
    v = np.zeros(len(perms), np.int32)
    vp = ctypes.c_void_p
    rc = native_lib.tdp_canonical(spi.ctypes.data_as(vp), ns.ctypes.data_as(vp), len(perms), sig.ctypes.data_as(vp),
                                  h.ctypes.data_as(vp), v.ctypes.data_as(vp))
    assert rc == 0
    return sig, h, v


def random_configurations(count, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for c in range(count):
        if c % 2 == 0:  # product of disjoint 3-cycles, like the proof's configurations
            m = int(rng.integers(1, 22))
            q = rng.permutation(3 * m)
            p = list(range(3 * m))
            for t in range(m):
                a, b, d = (int(x) for x in q[3 * t:3 * t + 3])
                p[a], p[b], p[d] = b, d, a
        else:  # cycles of mixed lengths >= 2
            n = int(rng.integers(2, 64))
            q = [int(x) for x in rng.permutation(n)]
            p = list(range(n))
            i = 0
            while i < n:
                L = int(rng.integers(2, 8))
                if n - i - L == 1 or i + L > n:
                    L = n - i
                cyc = q[i:i + L]
                for k, x in enumerate(cyc):
                    p[x] = cyc[(k + 1) % len(cyc)]
                i += L
        out.append(p)
    return out


def test_golden_configurations(native_lib, oracle):
    perms = [oracle.parse_cycles(rec["spi"]) for rec in GOLDEN]
    sig, h, _ = run(native_lib, perms)
    for r, rec in enumerate(GOLDEN):
        n = len(perms[r])
        assert np.array_equal(sig[r, :n], np.array(rec["canonical_signature"], np.float32))
        assert int(h[r]) == rec["hash_code"]


def test_random_configurations_match_oracle(native_lib, oracle):
    perms = random_configurations(3000, 1375)
    sig, h, v = run(native_lib, perms)
    for r, p in enumerate(perms):
        want_sig, want_h, want_v = oracle.canonical(p)
        n = len(p)
        assert np.array_equal(sig[r, :n], np.array(want_sig, np.float32)), r
        assert int(h[r]) == want_h and int(v[r]) == want_v, r
        assert not sig[r, n:].any()


def test_sortings_table_keys_match_oracle_hash(native_lib, oracle):
    """casefile.sortings_table keys the reference's case records by Configuration.hashCode
    (as AbstractSbtAlgorithm.loadSortings does)."""
    from tdp1375_b200 import casefile
    recs = []
    for name in ("cases_3_2.json", "cases_comb.json"):
        data = json.load(open(os.path.join(ROOT, "tests", "golden", name)))["records"]
        recs += [(r["spi"], [tuple(m) for m in r["moves"]]) for r in data]
    table = casefile.sortings_table(recs)
    assert sum(len(v) for v in table.values()) == len(recs)
    for h, group in table.items():
        for spi, _ in group:
            assert oracle.canonical(spi)[1] == h
