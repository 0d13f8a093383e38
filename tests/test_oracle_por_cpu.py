"""The partial-order reduction of commuting moves never changes a verdict, checked on the CPU:
the oracle's restatement of it (oracle_search_gpu_rule with the commute bit, the same skip
rule as the engine's por_skip) must reproduce every verdict of the config-1 fixture, which
the oracle made without it (tests/golden/verdicts_config1.json: full sorting at depths 11
and 7, partial mode at depth 6).  Every sequence found under the reduction is replayed.
Runs on the host cores through a spawn pool; no GPU."""
import multiprocessing as mp
import os

from conftest import load_golden

SETTINGS = (("full11", 11, True), ("full7", 7, True), ("partial6", 6, False))
FULL11_CASES = 120  # depth-11 negatives cost seconds each on one core


def _check(args):
    case, key, depth, full, want = args
    from oracle import oracle as O
    from tdp1375_b200.cases import config_cases, MIN_RATE
    pi, spi, even, _ = next(config_cases(1, 1, start=case))
    st, moves, _ = O.search_gpu_rule(list(pi), list(spi), even, float(MIN_RATE), depth, full, dedup=True,
                                     tight=(key == "full11"), commute=True)
    ok = st == want
    if ok and st == 1:
        ok, _ = O.replay_positions(list(pi), list(spi), moves, even, float(MIN_RATE), full)
    return case, key, st, want, ok


def test_reduction_keeps_config1_verdicts():
    rows = load_golden("verdicts_config1.json")["cases"]
    jobs = []
    for r in rows:
        for key, depth, full in SETTINGS:
            if r[key] not in (0, 1) or (key == "full11" and r["case"] >= FULL11_CASES):
                continue
            jobs.append((r["case"], key, depth, full, r[key]))
    assert len(jobs) >= 2000
    with mp.get_context("spawn").Pool(max(1, min(32, os.cpu_count() or 1))) as pool:
        results = pool.map(_check, jobs, chunksize=8)
    bad = [r for r in results if not r[4]]
    assert not bad, bad[:5]
