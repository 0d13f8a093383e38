"""Generates tests/golden/verdicts_config1.json with the CPU oracle.

Seeded config-1 instances (3-permutations, m ~ U{4,5,6}, pi = identity, ratio 1.375)
solved by the oracle's restatement of the CUDA rule (oracle/tdp_oracle.cpp, transposition
table on) in three settings:
  full11   full sorting, max depth 11, with the verdict-preserving tight bound (needed to
           decide the exhaustive negatives within the node limit);
  full7    full sorting, max depth 7, reference rule only;
  partial6 partial mode (the proof generator's mode), max depth 6, reference rule only.
A verdict of -2 means the node limit was hit (the case is not used by the tests).
Runs on all cores with a spawn pool:
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
    for key, full, depth, tight in (("full11", True, 11, True), ("full7", True, 7, False),
                                    ("partial6", False, 6, False)):
        st, moves, (e, c) = O.search_gpu_rule(list(pi), list(spi), even, float(MIN_RATE), depth, full,
                                              dedup=True, tight=tight, node_limit=node_limit)
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
            "rule": "sorting_search.cu:321-362 (float32), transposition table on; full11 adds the tight bound",
            "cases": rows}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "verdicts_config1.json")
    with open(path, "w") as fh:
        json.dump(data, fh, separators=(",", ":"))
    for key in ("full11", "full7", "partial6"):
        vals = [r[key] for r in rows]
        print(key, {v: vals.count(v) for v in set(vals)})


if __name__ == "__main__":
    main()
