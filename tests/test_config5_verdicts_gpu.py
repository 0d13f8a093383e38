"""Config-5 verdicts (the learned order's held-out set: m = 8..10, partial mode, max depth
11, ratio 1.375) against the oracle's restatement of the CUDA rule, on the first 120 cases
of the seeded stream (tests/golden/verdicts_config5.json, made by make_verdicts_config5.py).
The engine runs them in plain order and again with an untrained order model installed,
whose arbitrary root order, and arbitrary first-level lists, must not change a verdict.
Every sequence found is replayed."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

R1375 = float(np.float32(2) / np.float32(1.375))


def test_config5_verdicts_match_oracle_in_any_root_order(native_lib, oracle):
    from tdp1375_b200 import GPUSortingSearch, make_instances, order_model, search_batch
    from tdp1375_b200.cases import config_cases
    rows = [r for r in load_golden("verdicts_config5.json")["cases"] if r[3] in (0, 1)]
    assert len(rows) >= 100
    stream = list(config_cases(5, max(r[0] for r in rows) + 1))
    cases = [stream[r[0]][:3] for r in rows]
    GPUSortingSearch(1, 1, 256 << 20, 1 << 26)
    try:
        inst = make_instances(cases, 11, False)
        plain = search_batch(0, inst, len(cases), R1375)
        model = order_model.OrderModel()  # random weights: an arbitrary order
        model.install(0, enable=True, levels=1)
        ordered = search_batch(0, inst, len(cases), R1375)
        native_lib.tdp_enable_order_model(0, 2)
        ordered2 = search_batch(0, inst, len(cases), R1375)
        assert native_lib.tdp_mlp_error() == 0
        for res in (plain, ordered, ordered2):
            for row, case, r in zip(rows, cases, res):
                assert r.status == row[3], row[0]
                if r.status == 1:
                    pos = [[r.positions[3 * d + t] for t in range(3)] for d in range(r.depth)]
                    ok, _ = oracle.replay_positions(list(case[0]), list(case[1]), pos, case[2], R1375, False)
                    assert ok, row[0]
    finally:
        GPUSortingSearch.destroySlots()
