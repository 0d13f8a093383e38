"""GPU parity tests of the search engine against the CPU oracle and the reference fixtures."""
import ctypes
import threading
import time

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

R1375 = float(np.float32(2) / np.float32(1.375))
R15 = float(np.float32(2) / np.float32(1.5))


def run_batch(cases, max_depth, full, rate, slot=0):
    from tdp1375_b200 import make_instances, search_batch
    inst = make_instances(cases, max_depth, full)
    return search_batch(slot, inst, len(cases), rate)


def positions(res):
    return [[res.positions[3 * d], res.positions[3 * d + 1], res.positions[3 * d + 2]] for d in range(res.depth)]


def test_drop_in_small_fixtures(gpu_searcher, oracle):
    for name, rate, depth in (("cases_3_2.json", R15, 3), ("cases_7cycle.json", R15, 4)):
        for rec in load_golden(name)["records"]:
            spi, pi = rec["spi"], rec["pi"]
            init = oracle.count_even(spi)
            moves = gpu_searcher.search(pi, spi, init, rate, depth, False)
            assert moves, rec
            e, _ = oracle.replay_symbols(pi, spi, moves)
            assert e - init > 0 and np.float32(e - init) / np.float32(len(moves)) >= np.float32(rate)


@pytest.mark.parametrize("depth_mode", ["own", "eleven"])
def test_comb_fixtures_found(gpu_searcher, oracle, depth_mode):
    """All 673 known positives of cases-comb.txt answer FOUND (partial mode) and every
    returned sequence replays within the ratio."""
    recs = load_golden("cases_comb.json")["records"]
    if depth_mode == "own":
        groups = {}
        for r in recs:
            groups.setdefault(len(r["moves"]), []).append(r)
    else:
        groups = {11: recs}
    for depth, rows in groups.items():
        cases = [(r["pi"], r["spi"], oracle.count_even(r["spi"])) for r in rows]
        res = run_batch(cases, depth, False, R1375)
        for (pi, spi, init), r in zip(cases, res):
            assert r.status == 1, (depth, spi)
            ok, _ = oracle.replay_positions(pi, spi, positions(r), init, R1375, False)
            assert ok and r.depth <= depth


def test_config1_verdicts_match_oracle(gpu_searcher, oracle):
    from tdp1375_b200.cases import config_cases
    data = load_golden("verdicts_config1.json")
    rows = data["cases"]
    n = max(r["case"] for r in rows) + 1
    cases = list(config_cases(1, n))
    for key, full, depth in (("full11", True, 11), ("full7", True, 7), ("partial6", False, 6)):
        sel = [r for r in rows if r[key] in (0, 1)]
        assert len(sel) > 50, key
        batch = [cases[r["case"]][:3] for r in sel]
        res = run_batch(batch, depth, full, R1375)
        for row, case, r in zip(sel, batch, res):
            assert r.status == row[key], (key, row["case"])
            if r.status == 1:
                ok, _ = oracle.replay_positions(list(case[0]), list(case[1]), positions(r), case[2], R1375, full)
                assert ok


@pytest.mark.parametrize("full,depth", [(False, 8), (True, 8)])
def test_engine_modes_keep_verdicts(gpu_searcher, oracle, full, depth):
    """Single-instance calls, batched calls, and the engine with the tight bound off, with
    every triple enumerated, with same-cycle pairs only, with pairs and same-cycle triples,
    or with instances in flight capped (64 warps per instance; a cap of one instance), all
    give the same verdicts."""
    from tdp1375_b200 import GPUSortingSearch, api, native
    from tdp1375_b200.cases import config_cases
    cases = [c[:3] for c in config_cases(1, 40)]
    batch = run_batch(cases, depth, full, R1375)
    cfg = api.engine_config(1)
    variants = []
    for tight, sparse, wpi in ((1, 0, 0), (0, 0, 0), (0, 1, 0), (1, 1, 0), (0, 2, 0), (1, 2, 64), (1, 2, 100000)):
        api.set_engine_config(1, native.EngineConfig(cfg.blocks_per_sm, cfg.poll_interval, tight, cfg.task_capacity,
                                                     cfg.time_limit_s, sparse, 0, wpi))
        try:
            variants.append(run_batch(cases, depth, full, R1375, slot=1))
        finally:
            api.set_engine_config(1, cfg)
    for idx, ((pi, spi, even), b) in enumerate(zip(cases, batch)):
        assert all(v[idx].status == b.status for v in variants), idx
        if idx < 10:
            pos = GPUSortingSearch.searchForSortingSeq(list(pi), list(spi), even, R1375, depth, full, 0)
            assert (1 if pos else 0) == b.status
        if b.status == 1:
            ok, _ = oracle.replay_positions(list(pi), list(spi), positions(b), even, R1375, full)
            assert ok


def test_edge_cases(gpu_searcher):
    from tdp1375_b200 import GPUSortingSearch
    for n in (0, 1, 2):
        assert GPUSortingSearch.searchForSortingSeq(list(range(n)), list(range(n)), n, R1375, 5, True, 0) == []
    ident = list(range(12))
    assert GPUSortingSearch.searchForSortingSeq(ident, ident, 12, R1375, 11, True, 0) == []
    with pytest.raises(RuntimeError, match="MAX_N"):
        GPUSortingSearch.searchForSortingSeq(list(range(64)), list(range(64)), 0, R1375, 5, True, 0)
    with pytest.raises(RuntimeError, match="maximumDepth"):
        GPUSortingSearch.searchForSortingSeq(ident, ident, 12, R1375, 16, True, 0)
    with pytest.raises(RuntimeError, match="maximumDepth"):
        GPUSortingSearch.searchForSortingSeq(ident, ident, 12, R1375, 0, True, 0)
    with pytest.raises(RuntimeError, match="permutation"):
        GPUSortingSearch.searchForSortingSeq(ident, [0] * 12, 12, R1375, 5, True, 0)
    with pytest.raises(RuntimeError, match="invalid slot"):
        GPUSortingSearch.searchForSortingSeq(ident, ident, 12, R1375, 5, True, 7)


def test_large_n_generic_layout(gpu_searcher, oracle):
    """n > 32 uses the two-words-per-lane layout: a 3-permutation on 63 symbols at depth 2."""
    from tdp1375_b200.cases import three_permutation
    rng = np.random.Generator(np.random.PCG64(5))
    for m in (11, 15, 21):
        pi, spi, even = three_permutation(m, rng)
        got = run_batch([(pi, spi, even)], 2, False, R1375)[0]
        want, _, _ = oracle.search_gpu_rule(list(pi), list(spi), even, R1375, 2, False)
        assert got.status == want
        if got.status == 1:
            ok, _ = oracle.replay_positions(list(pi), list(spi), positions(got), even, R1375, False)
            assert ok


def test_cancel_stops_a_long_search(gpu_searcher):
    from tdp1375_b200 import GPUSortingSearch
    from tdp1375_b200.cases import three_permutation
    rng = np.random.Generator(np.random.PCG64(11))
    pi, spi, even = three_permutation(10, rng)  # full sorting at depth 14: a long exhaustive search
    errors = []

    def worker():
        try:
            GPUSortingSearch.searchForSortingSeq(list(pi), list(spi), even, float(np.float32(2) / np.float32(1.45)),
                                                 14, True, 1)
            errors.append("finished")
        except RuntimeError as exc:
            errors.append(str(exc))

    t = threading.Thread(target=worker)
    t.start()
    time.sleep(0.5)
    GPUSortingSearch.cancelSort(1)
    t.join(60)
    assert not t.is_alive()
    assert errors and (errors[0] == "GPU sorting search cancelled" or errors[0] == "finished")
    # the slot is usable afterwards
    assert GPUSortingSearch.searchForSortingSeq(list(range(5)), list(range(5)), 5, R1375, 3, True, 1) == []


def test_cuda_graph_replay_matches_direct_launch(gpu_searcher, oracle):
    """tdp_batch_run with use_cuda_graph replays one captured graph (root ordering off):
    two replays give the verdicts of a direct launch, with fresh table generations."""
    import ctypes
    from tdp1375_b200 import api, make_instances, native
    from tdp1375_b200.cases import config_cases
    lib = native.load()
    cases = [c[:3] for c in config_cases(1, 48)]
    inst = make_instances(cases, 11, True)
    direct = run_batch(cases, 11, True, R1375, slot=1)
    cfg = api.engine_config(1)
    graph_cfg = native.EngineConfig(cfg.blocks_per_sm, cfg.poll_interval, cfg.tight_bound, cfg.task_capacity,
                                    cfg.time_limit_s, cfg.sparse_enumeration, 1)
    api.set_engine_config(1, graph_cfg)
    try:
        assert lib.tdp_batch_prepare(1, inst, len(cases), ctypes.c_float(R1375)) == 0, native.last_error()
        for _ in range(2):
            assert lib.tdp_batch_run(1) == 0, native.last_error()
            res = (native.Result * len(cases))()
            assert lib.tdp_batch_results(1, res) == 0
            assert [r.status for r in res] == [r.status for r in direct]
            for (pi, spi, even), r in zip(cases, res):
                if r.status == 1:
                    ok, _ = oracle.replay_positions(list(pi), list(spi), positions(r), even, R1375, True)
                    assert ok
    finally:
        api.set_engine_config(1, cfg)
