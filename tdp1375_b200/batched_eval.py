"""Batched uneven search: one persistent, graph-captured launch over many instances.

    python -m tdp1375_b200.batched_eval [--count 1000000] [--sample 100000] [--out result.json]

Instances come from the seeded uneven generator: 3-permutations with m truncated-geometric
on 3..10 (p = 0.35) mixed with 10% random permutations of n' = 20..30 (pi = 0 followed by a
shuffle, spi = sigma o pi^-1).  They are searched in partial mode (the proof generator's
mode) with ratio 1.375 and max depth 11.  The autotuner first times its candidate
configurations (poll interval, warps per instance, table size) on a sample; the chosen one
is installed, with the transposition table raised to --run-table-entries (2^31 entries,
64 GB) for the full run.  Then the full set is uploaded
once (tdp_batch_prepare), run through a captured CUDA graph (tdp_batch_run with
use_cuda_graph), and read back.  The device time of the run is reported.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

from . import api, autotune, native
from .cases import MIN_RATE, config_cases


WORKLOAD = "batched-partial-d11"
STAT_FIELDS = ("nodes", "children", "dedup_probes", "dedup_pruned", "dedup_inserts", "dedup_full", "donations",
               "busy_warp_cycles", "warp_cycles")


def instances(count: int):
    cases, ms = [], []
    for pi, spi, even, m in config_cases(4, count):
        cases.append((pi, spi, even))
        ms.append(m)
    return cases, ms


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--count", type=int, default=1_000_000)
    p.add_argument("--sample", type=int, default=100_000)
    p.add_argument("--table-entries", type=int, default=1 << 30)
    p.add_argument("--depth", type=int, default=11)
    p.add_argument("--tune-cache", default="")
    p.add_argument("--run-table-entries", type=int, default=(1 << 31) - 1,
                   help="table for the full run when larger than the tuned one (rounded up to a power of two; "
                        "the C ABI takes an int)")
    p.add_argument("--time-limit-s", type=float, default=600.0)
    p.add_argument("--use-cached", action="store_true", help="reuse a cached autotune choice when present")
    p.add_argument("--out", default="")
    args = p.parse_args(argv)
    rate = float(MIN_RATE)
    lib = native.load()

    t0 = time.perf_counter()
    cases, ms = instances(args.count)
    t_gen = time.perf_counter() - t0
    inst = api.make_instances(cases, args.depth, False)

    cache_path = args.tune_cache or autotune.CACHE
    choice = autotune.cached(WORKLOAD, cache_path) if args.use_cached else None
    if choice is not None and "warps_per_instance" not in choice:
        choice = None  # cached before this tunable existed
    if choice is None:
        sample = api.make_instances(cases[: args.sample], args.depth, False)
        space = {"poll_interval": [16, 32, 64], "sparse_enumeration": [2], "warps_per_instance": [0, 4, 8]}
        choice = autotune.tune(WORKLOAD, sample, min(args.sample, len(cases)), rate,
                               table_sizes=(1 << 28, args.table_entries), space=space, cache_path=cache_path)

    print(json.dumps({"phase": "tuned", "generation_s": round(t_gen, 2), "choice": choice}), flush=True)
    # A sample cannot show the live-entry load of the full run (thousands of long instances
    # in flight for minutes), so the full run takes the larger of the tuned table and
    # --run-table-entries.
    entries = max(choice["table_entries"], args.run_table_entries)
    api.GPUSortingSearch(1, 1, 3000 << 20, entries)
    try:
        autotune.apply(0, choice)
        cfg = api.engine_config(0)
        cfg.use_cuda_graph = 1
        cfg.time_limit_s = args.time_limit_s
        api.set_engine_config(0, cfg)
        t0 = time.perf_counter()
        if lib.tdp_batch_prepare(0, inst, len(cases), ctypes.c_float(rate)) != 0:
            raise RuntimeError(native.last_error())
        t_prep = time.perf_counter() - t0
        if lib.tdp_batch_run(0) != 0:
            err = native.last_error()
            st = api.last_stats(0)
            print(json.dumps({"phase": "run failed", "error": err, "kernel_ms": st.kernel_ms,
                              "stats": {f: int(getattr(st, f)) for f in STAT_FIELDS}}), flush=True)
            raise RuntimeError(err)
        st = api.last_stats(0)
        res = (native.Result * len(cases))()
        lib.tdp_batch_results(0, res)
        status = np.array([r.status for r in res])
        nodes = np.array([r.nodes for r in res], dtype=np.int64)
        ms_arr = np.array(ms)
        per_m = {}
        for m in sorted(set(ms)):
            sel = ms_arr == m
            per_m[str(m) if m else "random"] = {"count": int(sel.sum()), "found": int((status[sel] == 1).sum()),
                                                "mean_nodes": float(nodes[sel].mean())}
        out = {
            "instances": len(cases), "generation_s": round(t_gen, 2), "prepare_s": round(t_prep, 2),
            "kernel_ms": st.kernel_ms, "cases_per_s": len(cases) / (st.kernel_ms / 1e3),
            "nodes": int(st.nodes), "nodes_per_s": st.nodes / (st.kernel_ms / 1e3), "children": int(st.children),
            "launches": st.launches, "graph": True, "autotune_choice": choice, "table_entries": 1 << (entries - 1).bit_length(),
            "stats": {f: int(getattr(st, f)) for f in STAT_FIELDS},
            "found": int((status == 1).sum()), "not_found": int((status == 0).sum()),
            "other": int(((status != 0) & (status != 1)).sum()), "per_m": per_m,
        }
        print(json.dumps(out), flush=True)
        if args.out:
            with open(args.out, "w") as fh:
                json.dump(out, fh, indent=1)
    finally:
        api.GPUSortingSearch.destroySlots()


if __name__ == "__main__":
    main()
