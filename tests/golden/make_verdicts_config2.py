"""Generates tests/golden/verdicts_config2.json with the CPU oracle.

Config-2 instances (3-permutations, m ~ U{4..8}, pi = identity, ratio 1.375) from the start
of the seeded stream, in the bench's setting: full sorting, max depth 11.  They are solved by
the oracle's restatement of the CUDA rule (oracle/tdp_oracle.cpp) with the transposition
table and the verdict-preserving tight bound.  Cases with m = 8 are left out: an exhaustive
m = 8 negative takes tens of millions of nodes on one core.  A verdict of -2 means the node
limit was hit (the case is not used by the tests).  Runs on all cores with a spawn pool:
    python tests/golden/make_verdicts_config2.py [scan] [node_limit] [start]
With start > 0 the cases [start, start + scan) are solved and merged into the existing file.
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
    pi, spi, even, m = next(config_cases(2, 1, start=case))
    if m > 7:
        return None
    st, _, (e, _) = O.search_gpu_rule(list(pi), list(spi), even, float(MIN_RATE), 11, True, dedup=True, tight=True,
                                      node_limit=node_limit)
    return {"case": case, "m": m, "full11": st, "nodes": e}


def main():
    scan = int(sys.argv[1]) if len(sys.argv) > 1 else 6250
    node_limit = int(sys.argv[2]) if len(sys.argv) > 2 else 20_000_000
    start = int(sys.argv[3]) if len(sys.argv) > 3 else 0
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "verdicts_config2.json")
    ctx = mp.get_context("spawn")
    with ctx.Pool(os.cpu_count()) as pool:
        rows = [r for r in pool.map(solve, [(c, node_limit) for c in range(start, start + scan)], chunksize=4)
                if r is not None]
    if start > 0:
        old = json.load(open(path))
        if old["scanned"] != start or old["node_limit"] != node_limit:
            raise SystemExit("the existing file must cover exactly [0, start) with the same node limit")
        rows = old["cases"] + rows
    data = {"config": 2, "min_rate": "float32(2)/float32(1.375)", "node_limit": node_limit, "scanned": start + scan,
            "rule": "sorting_search.cu:321-362 (float32), full sorting, depth 11, transposition table and tight bound",
            "cases": rows}
    with open(path, "w") as fh:
        json.dump(data, fh, separators=(",", ":"))
    vals = [r["full11"] for r in rows]
    print(len(rows), {v: vals.count(v) for v in set(vals)})


if __name__ == "__main__":
    main()
