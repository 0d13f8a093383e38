"""Generates tests/golden/verdicts_config1.json with the CPU oracle.

Seeded config-1 instances (3-permutations, m ~ U{4,5,6}, pi = identity, full sorting,
ratio 1.375, max depth 11) solved by the oracle's restatement of the CUDA rule
(oracle/tdp_oracle.cpp, transposition table on).  Cases that exceed the node limit are
left out (listed as "skipped").  Also records partial-mode verdicts at depth 6 for the same
instances.  Runs on all cores with a spawn pool:
    python tests/golden/make_verdicts.py [count] [node_limit]
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def solve(args):
    case, node_limit = args
    import numpy as np
    from oracle import oracle as O
    from tdp1375_b200.cases import config_cases, MIN_RATE
    pi, spi, even, m = next(config_cases(1, 1, start=case))
    out = {"case": case, "m": m}
    for key, full, depth in (("full11", True, 11), ("partial6", False, 6)):
        st, moves, (e, c) = O.search_gpu_rule(list(pi), list(spi), even, float(MIN_RATE), depth, full,
                                              dedup=True, tight=False, node_limit=node_limit)
        out[key] = st
        out[key + "_nodes"] = e
    return out


def main():
    count = int(sys.argv[1]) if len(sys.argv) > 1 else 400
    node_limit = int(sys.argv[2]) if len(sys.argv) > 2 else 400000
    ctx = mp.get_context("spawn")
    with ctx.Pool(os.cpu_count()) as pool:
        rows = pool.map(solve, [(c, node_limit) for c in range(count)], chunksize=1)
    data = {"config": 1, "min_rate": "float32(2)/float32(1.375)", "node_limit": node_limit,
            "rule": "sorting_search.cu:321-362 (float32), transposition table on, tight bound off",
            "cases": rows}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "verdicts_config1.json")
    with open(path, "w") as fh:
        json.dump(data, fh, separators=(",", ":"))
    full = [r["full11"] for r in rows]
    part = [r["partial6"] for r in rows]
    print("full11", {v: full.count(v) for v in set(full)}, "partial6", {v: part.count(v) for v in set(part)})


if __name__ == "__main__":
    main()
