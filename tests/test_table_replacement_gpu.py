"""A transposition table far smaller than the searches need must give the verdicts of the
fixtures under every full-window policy (tdp_engine_config.table_replacement): admit
without recording, as sorting_search.cu:291-297 does, or overwrite a live entry (the
deepest, the oldest, or the oldest of the deepest) while other warps read it, their key
reads validated by the version carried in each key word.  Also: the per-launch device
deadline ends a long search with TDP_ERR_DEVICE and leaves the slot usable."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

R1375 = float(np.float32(2) / np.float32(1.375))


def _config(slot, **changes):
    from tdp1375_b200 import api
    cfg = api.engine_config(slot)
    for k, v in changes.items():
        setattr(cfg, k, v)
    api.set_engine_config(slot, cfg)


def test_tiny_table_keeps_verdicts_under_every_replacement_policy(native_lib, oracle):
    from tdp1375_b200 import GPUSortingSearch, api, make_instances, search_batch
    from tdp1375_b200.cases import config_cases
    rows = [r for r in load_golden("verdicts_config2.json")["cases"] if r["full11"] in (0, 1)]
    # the heaviest searches of the fixture's first part plus every found case among them
    head = [r for r in rows if r["case"] < 1200]
    heavy = sorted(head, key=lambda r: -r["nodes"])[:40]
    found = [r for r in head if r["full11"] == 1][:60]
    sel = sorted({r["case"]: r for r in heavy + found}.values(), key=lambda r: r["case"])
    stream = list(config_cases(2, max(r["case"] for r in sel) + 1))
    cases = [stream[r["case"]][:3] for r in sel]
    GPUSortingSearch(1, 1, 256 << 20, 1 << 14)  # 16,384 entries: windows fill at once
    try:
        for policy in (0, 1, 2, 3):
            _config(0, table_replacement=policy)
            res = search_batch(0, make_instances(cases, 11, True), len(cases), R1375)
            st = api.last_stats(0)
            if policy:
                assert st.dedup_replaced > 0
            else:
                assert st.dedup_replaced == 0 and st.dedup_full > 0
            for row, case, r in zip(sel, cases, res):
                assert r.status == row["full11"], (policy, row["case"])
                if r.status == 1:
                    pos = [[r.positions[3 * d + t] for t in range(3)] for d in range(r.depth)]
                    ok, _ = oracle.replay_positions(list(case[0]), list(case[1]), pos, case[2], R1375, True)
                    assert ok, (policy, row["case"])
    finally:
        GPUSortingSearch(1, 2, 256 << 20, 1 << 21)  # the slots the session fixture set up


def test_device_deadline_returns_device_error_and_slot_survives(native_lib):
    from tdp1375_b200 import GPUSortingSearch, api
    from tdp1375_b200.cases import config_cases
    GPUSortingSearch(1, 2, 256 << 20, 1 << 21)
    case = next(c for c in config_cases(2, 50) if c[3] == 8)  # an m = 8 full-sorting search takes seconds
    cfg = api.engine_config(1)
    _config(1, time_limit_s=0.002)
    try:
        with pytest.raises(RuntimeError, match="device time limit"):
            GPUSortingSearch.searchForSortingSeq(list(case[0]), list(case[1]), case[2], R1375, 11, True, 1)
    finally:
        api.set_engine_config(1, cfg)
    # the same slot answers the next call normally
    assert GPUSortingSearch.searchForSortingSeq(list(range(6)), list(range(6)), 6, R1375, 4, True, 1) == []
    small = next(config_cases(1, 1))
    got = GPUSortingSearch.searchForSortingSeq(list(small[0]), list(small[1]), small[2], R1375, 11, True, 1)
    want = load_golden("verdicts_config1.json")["cases"][0]["full11"]
    assert (1 if got else 0) == want


def test_engine_options_keep_config1_verdicts(native_lib, oracle):
    """The partial-order reduction (commute) and probe-free leaf admission (probe_leaves = 0)
    on and off, on the config-1 fixture's full-sorting and partial settings."""
    from tdp1375_b200 import GPUSortingSearch, api, make_instances, search_batch
    from tdp1375_b200.cases import config_cases
    rows = load_golden("verdicts_config1.json")["cases"][:250]
    stream = list(config_cases(1, len(rows)))
    GPUSortingSearch(1, 1, 256 << 20, 1 << 22)
    try:
        for commute, probe_leaves in ((1, 0), (0, 0), (1, 1), (0, 1)):
            _config(0, commute=commute, probe_leaves=probe_leaves)
            for key, full, depth in (("full11", True, 11), ("partial6", False, 6)):
                sel = [r for r in rows if r[key] in (0, 1)]
                cases = [stream[r["case"]][:3] for r in sel]
                res = search_batch(0, make_instances(cases, depth, full), len(cases), R1375)
                st = api.last_stats(0)
                assert (st.commute_skips > 0) == bool(commute) or key == "partial6"
                for row, case, r in zip(sel, cases, res):
                    assert r.status == row[key], (commute, probe_leaves, key, row["case"])
                    if r.status == 1:
                        pos = [[r.positions[3 * d + t] for t in range(3)] for d in range(r.depth)]
                        ok, _ = oracle.replay_positions(list(case[0]), list(case[1]), pos, case[2], R1375, full)
                        assert ok
    finally:
        GPUSortingSearch(1, 2, 256 << 20, 1 << 21)
