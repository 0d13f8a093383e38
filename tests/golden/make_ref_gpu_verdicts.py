"""Generates tests/golden/ref_gpu_verdicts_config<c>.json with the reference's own CUDA search.

The reference kernel (sorting_search.cu + slot_manager.cu, compiled from the reference
sources by `make -C oracle ref` into oracle/_ref/libtdp_ref.so, driven without JNI by
oracle/ref_harness.cu) runs the seeded instances of one BASELINE configuration on a B200,
one performGpuSortingSearch call per case, as GPUSortingSearch does.  Each row is
[case, m, verdict, depth, milliseconds]: verdict 1 found, 0 not found, 2 the case hit the
per-case time limit (the harness then cancels it through cancelGpuSort), 3 the reference
reported a queue overflow.  Every sequence found is replayed with the oracle before it is
recorded.  Rows of an existing output file are kept, so the script resumes where a previous
run stopped:

    python tests/golden/make_ref_gpu_verdicts.py --config 2 --count 5000 --table-entries 2097152 \
        --timeout-s 60 --budget-s 1800 [--only-m 8] [--out PATH]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--config", type=int, default=2)
    p.add_argument("--start", type=int, default=0)
    p.add_argument("--count", type=int, default=5000)
    p.add_argument("--max-depth", type=int, default=11)
    p.add_argument("--partial", action="store_true", help="fullSorting = false (the proof generator's mode)")
    p.add_argument("--table-entries", type=int, default=1 << 21)
    p.add_argument("--queue-mb", type=int, default=3000)
    p.add_argument("--timeout-s", type=float, default=60.0)
    p.add_argument("--budget-s", type=float, default=1800.0)
    p.add_argument("--only-m", type=int, default=0)
    p.add_argument("--out", default="")
    args = p.parse_args()
    from oracle import oracle as O
    from oracle import reference_gpu as R
    from tdp1375_b200.cases import config_cases, MIN_RATE

    full = not args.partial
    out = args.out or os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                   f"ref_gpu_verdicts_config{args.config}.json")
    meta = {"config": args.config, "min_rate": "float32(2)/float32(1.375)", "max_depth": args.max_depth,
            "full_sorting": full, "table_entries": args.table_entries, "queue_bytes": args.queue_mb << 20,
            "slots": 1, "timeout_s": args.timeout_s,
            "source": "reference sorting_search.cu:701-856 (performGpuSortingSearch) on one B200, built by "
                      "oracle/Makefile (ref) and driven by oracle/ref_harness.cu",
            "columns": ["case", "m", "verdict (1 found, 0 not found, 2 time limit, 3 overflow)", "depth", "ms"]}
    rows = {}
    if os.path.exists(out):
        old = json.load(open(out))
        for k in ("config", "max_depth", "full_sorting"):
            if old[k] != meta[k]:
                raise SystemExit(f"{out} was made with another {k}")
        # a case decided under any table size keeps its verdict; a timed-out case is retried
        rows = {r[0]: r for r in old["rows"] if r[2] in (0, 1)}
    R.init(1, 1, args.queue_mb << 20, args.table_entries)
    t0 = time.time()
    done = 0
    try:
        for case, (pi, spi, even, m) in zip(range(args.start, args.start + args.count),
                                            config_cases(args.config, args.count, start=args.start)):
            if case in rows or (args.only_m and m != args.only_m):
                continue
            if time.time() - t0 > args.budget_s:
                break
            st, moves, ms = R.search(list(pi), list(spi), even, float(MIN_RATE), args.max_depth, full,
                                     timeout_s=args.timeout_s)
            if st == R.FOUND:
                ok, _ = O.replay_positions(list(pi), list(spi), moves, even, float(MIN_RATE), full)
                if not ok:
                    raise SystemExit(f"case {case}: the reference's sequence does not replay")
            rows[case] = [case, m, st, len(moves), round(ms, 2)]
            done += 1
            if done % 50 == 0:
                print(f"{done} cases in {time.time() - t0:.0f} s", flush=True)
    finally:
        R.destroy()
        meta["rows"] = [rows[c] for c in sorted(rows)]
        with open(out, "w") as fh:
            json.dump(meta, fh, separators=(",", ":"))
    vals = [r[2] for r in meta["rows"]]
    print(json.dumps({"rows": len(vals), "verdicts": {v: vals.count(v) for v in sorted(set(vals))},
                      "elapsed_s": round(time.time() - t0, 1)}))


if __name__ == "__main__":
    main()
