"""Generates tests/golden/verdicts_config5.json with the CPU oracle.

Config-5 instances (the held-out evaluation set of the learned order: 3-permutations with
m uniform in 8..10) from the start of the seeded stream, in the evaluation's setting:
partial mode, ratio 1.375, max depth 11.  They are solved by the oracle's restatement of
the CUDA rule (oracle/tdp_oracle.cpp) with the transposition table and the
verdict-preserving tight bound.  A verdict of -2 means the node limit was hit (the case
is not used by the tests).
    python tests/golden/make_verdicts_config5.py [scan] [node_limit]
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
    from oracle import oracle as O
    from tdp1375_b200.cases import config_cases, MIN_RATE
    pi, spi, even, m = next(config_cases(5, 1, start=case))
    st, _, (e, _) = O.search_gpu_rule(list(pi), list(spi), even, float(MIN_RATE), 11, False, dedup=True, tight=True,
                                      node_limit=node_limit)
    return [case, m, len(pi), st]


def main():
    scan = int(sys.argv[1]) if len(sys.argv) > 1 else 120
    node_limit = int(sys.argv[2]) if len(sys.argv) > 2 else 2_000_000
    ctx = mp.get_context("spawn")
    with ctx.Pool(os.cpu_count()) as pool:
        rows = [r for r in pool.map(solve, [(c, node_limit) for c in range(scan)], chunksize=2) if r is not None]
    data = {"config": 5, "min_rate": "float32(2)/float32(1.375)", "node_limit": node_limit, "scanned": scan,
            "rule": "sorting_search.cu:321-362 (float32), partial mode, depth 11, transposition table and tight bound",
            "columns": ["case", "m", "n", "partial11 verdict"], "cases": rows}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "verdicts_config5.json")
    with open(path, "w") as fh:
        json.dump(data, fh, separators=(",", ":"))
    vals = [r[3] for r in rows]
    print(len(rows), {v: vals.count(v) for v in set(vals)})


if __name__ == "__main__":
    main()
