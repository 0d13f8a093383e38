"""Config-4 verdicts in the batched run's setting (partial mode, max depth 11, ratio 1.375)
against the oracle's restatement of the CUDA rule: the m < 8 cases among the first 6,000
of the seeded stream, random permutations of n' = 20..30 included
(tests/golden/verdicts_config4.json, made by make_verdicts_config4.py).  They run as one
batch through a captured CUDA graph, and every sequence found is replayed on the host."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

R1375 = float(np.float32(2) / np.float32(1.375))


def test_config4_verdicts_match_oracle(native_lib, oracle):
    from tdp1375_b200 import GPUSortingSearch, api, make_instances, native
    from tdp1375_b200.cases import config_cases
    rows = [r for r in load_golden("verdicts_config4.json")["cases"] if r[3] in (0, 1)]
    assert len(rows) > 5000 and sum(1 for r in rows if r[1] == 0) > 500
    stream = list(config_cases(4, max(r[0] for r in rows) + 1))
    cases = [stream[r[0]][:3] for r in rows]
    GPUSortingSearch(1, 1, 256 << 20, 1 << 26)
    try:
        cfg = api.engine_config(0)
        cfg.use_cuda_graph = 1
        api.set_engine_config(0, cfg)
        lib = native.load()
        assert lib.tdp_batch_prepare(0, make_instances(cases, 11, False), len(cases), ctypes.c_float(R1375)) == 0
        assert lib.tdp_batch_run(0) == 0, native.last_error()
        res = (native.Result * len(cases))()
        lib.tdp_batch_results(0, res)
        for row, case, r in zip(rows, cases, res):
            assert r.status == row[3], row[0]
            if r.status == 1:
                pos = [[r.positions[3 * d + t] for t in range(3)] for d in range(r.depth)]
                ok, _ = oracle.replay_positions(list(case[0]), list(case[1]), pos, case[2], R1375, False)
                assert ok, row[0]
    finally:
        GPUSortingSearch.destroySlots()
