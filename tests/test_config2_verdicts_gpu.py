"""Config-2 verdicts in the bench's setting (full sorting, max depth 11, ratio 1.375) against
the oracle's restatement of the CUDA rule, on the m <= 7 cases at the start of the seeded
stream (tests/golden/verdicts_config2.json, made by make_verdicts_config2.py).  Every
sequence found is replayed on the host."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

R1375 = float(np.float32(2) / np.float32(1.375))


def test_config2_verdicts_match_oracle(native_lib, oracle):
    from tdp1375_b200 import GPUSortingSearch, make_instances, search_batch
    from tdp1375_b200.cases import config_cases
    rows = [r for r in load_golden("verdicts_config2.json")["cases"] if r["full11"] in (0, 1)]
    assert len(rows) > 250
    n = max(r["case"] for r in rows) + 1
    stream = list(config_cases(2, n))
    cases = [stream[r["case"]][:3] for r in rows]
    # a table large enough for hundreds of exhaustive searches in flight
    GPUSortingSearch(1, 1, 256 << 20, 1 << 28)
    try:
        res = search_batch(0, make_instances(cases, 11, True), len(cases), R1375)
        for row, case, r in zip(rows, cases, res):
            assert r.status == row["full11"], row["case"]
            if r.status == 1:
                pos = [[r.positions[3 * d + t] for t in range(3)] for d in range(r.depth)]
                ok, _ = oracle.replay_positions(list(case[0]), list(case[1]), pos, case[2], R1375, True)
                assert ok, row["case"]
    finally:
        GPUSortingSearch.destroySlots()
