"""CPU pin of the oracle's configuration signatures against the reference's own golden
values (ConfigurationTest.java, extracted to tests/golden/configuration_golden.json)."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "configuration_golden.json")))["configurations"]


def f32(xs):
    return np.array(xs, dtype=np.float32)


@pytest.mark.parametrize("rec", GOLDEN, ids=[r["spi"] for r in GOLDEN])
def test_signature_canonical_and_hash_match_reference(oracle, rec):
    spi = oracle.parse_cycles(rec["spi"])
    assert np.array_equal(f32(oracle.signature(spi)), f32(rec["signature"]))
    sig, h, _ = oracle.canonical(spi)
    assert np.array_equal(f32(sig), f32(rec["canonical_signature"]))
    assert h == rec["hash_code"]
    assert oracle.signature_hash(sig) == rec["hash_code"]


@pytest.mark.parametrize("rec", GOLDEN, ids=[r["spi"] for r in GOLDEN])
def test_equivalent_signatures_match_reference_set(oracle, rec):
    spi = oracle.parse_cycles(rec["spi"])
    got = {tuple(f32(s).tolist()) for s in oracle.equivalent_signatures(spi)}
    want = {tuple(f32(s).tolist()) for s in rec["equivalent_signatures"]}
    assert len(oracle.equivalent_signatures(spi)) == len(rec["equivalent_signatures"])
    assert got == want
