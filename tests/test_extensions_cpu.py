"""Extension step of the proof generator (Extensions.java): signatures against the oracle,
Configuration.ofSignature round trips, open gates against ConfigurationTest, and the
structure of every Type 1/2/3 extension."""
import json
import os
import random

import numpy as np
import pytest

from conftest import ROOT
from tdp1375_b200 import extensions as X

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "configuration_golden.json")))["configurations"]
OPEN_GATES = {"(0 9 7)(1 5 2 6 3)(4 10 8)": set(), "(0 8 2)(1 6 4)(3 7 5)": {0},
              "(0 5 1 11 3)(2 12 9 8 4)(6 10 7)": {7, 9}}  # ConfigurationTest.java:26-29, 107-110, 184-187


def random_configuration(rng, n):
    q = list(range(n))
    rng.shuffle(q)
    p = list(range(n))
    i = 0
    while i < n:
        L = rng.choice([3, 3, 3, 5, 2, 4])
        if n - i - L < 2 or i + L > n:
            L = n - i
        cyc = q[i:i + L]
        for k, x in enumerate(cyc):
            p[x] = cyc[(k + 1) % len(cyc)]
        i += L
    return p


def test_signature_matches_oracle_and_round_trips(oracle):
    rng = random.Random(8)
    for _ in range(300):
        spi = random_configuration(rng, rng.randint(3, 40))
        sig = X.signature(spi)
        assert np.array_equal(np.float32(sig), np.float32(oracle.signature(spi)))
        back = X.of_signature(sig)
        assert np.array_equal(np.float32(X.signature(back)), np.float32(sig))


@pytest.mark.parametrize("rec", GOLDEN, ids=[r["spi"] for r in GOLDEN])
def test_open_gates_match_reference(oracle, rec):
    spi = oracle.parse_cycles(rec["spi"])
    assert X.open_gates(spi) == OPEN_GATES[rec["spi"]]
    # ofSignature(signature) round trip of ConfigurationTest.testSignatureRoundTrip
    assert np.array_equal(np.float32(X.signature(X.of_signature(rec["signature"]))), np.float32(rec["signature"]))


def cycle_lengths(spi):
    return sorted(len(c) for c in X.cycles_in_order(spi))


@pytest.mark.parametrize("rec", GOLDEN, ids=[r["spi"] for r in GOLDEN])
def test_extension_structure(oracle, rec):
    spi = oracle.parse_cycles(rec["spi"])
    n, lengths = len(spi), cycle_lengths(spi)
    gates = X.open_gates(spi)
    t1 = X.type1_extensions(spi)
    assert len(t1) == len(gates) * (n * (n + 1) // 2 - 1)
    t2 = X.type2_extensions(spi)
    assert len(t2) == (0 if gates else (n + 2) * (n + 1) * n // 6 - n)
    for _, ext in t1 + t2:  # one new 3-cycle
        assert sorted(ext) == list(range(n + 3)) and cycle_lengths(ext) == sorted(lengths + [3])
    for desc, ext in X.type3_extensions(spi):  # one cycle grown by two symbols
        assert sorted(ext) == list(range(n + 2))
        grown = cycle_lengths(ext)
        assert len(grown) == len(lengths) and sum(grown) == n + 2
        if "turn oriented" in desc:
            assert 5 in grown and 3 in lengths


@pytest.mark.parametrize("rec", GOLDEN, ids=[r["spi"] for r in GOLDEN])
def test_combination_extensions_structure(oracle, rec):
    spi = oracle.parse_cycles(rec["spi"])
    n, lengths = len(spi), cycle_lengths(spi)
    out = X.combination_extensions(spi)
    assert len(out) == len(X.BAD_SMALL_COMPONENTS) * n
    for desc, ext in out:
        b = int(desc.split()[0].split("=")[1])
        comp = X._successor_of(X.BAD_SMALL_COMPONENTS[b])
        assert sorted(ext) == list(range(n + len(comp)))
        assert cycle_lengths(ext) == sorted(lengths + cycle_lengths(comp))
