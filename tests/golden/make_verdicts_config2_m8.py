"""Generates tests/golden/verdicts_config2_m8.json: the Java CPU rule's verdicts on the m = 8
cases of config 2, computed by the CPU oracle.

For 3-permutations with m = 8 (n = 24) in full-sorting mode at max depth 11, the CPU search
(SortingSearch.java:55-70, double precision) and the CUDA rule (sorting_search.cu:333-349,
float) differ only at nodes whose best-case final depth k = depth + ceil((n - even)/2) is
11: there the optimistic gain is exactly 16, which passes ceilf(1.4545455f * 11) = 16 but
not Math.ceil(1.454545497894287 * 11) = 17.  Along any move sequence k never decreases
(a move changes the odd-cycle count by at most 2), and the node before the last move of a
sorting of length L has k = L, so the CPU rule finds exactly the sortings of length <= 10,
while the CUDA rule also finds those of length 11.  Both rules admit every node with k <= 10
(the optimistic gain 38 - 2k >= ceil(1.4545 k) there), so the CPU rule's verdict at depth 11
equals the CUDA rule's verdict at depth 10.  This script computes the latter with the
oracle's restatement of the CUDA rule (transposition table and the verdict-preserving tight
bound), one case per core:

    python tests/golden/make_verdicts_config2_m8.py [scan] [node_limit]

Rows: [case, verdict at depth 10 (the CPU rule's verdict at 11), expanded nodes]; -2 marks
the node limit.  A case whose CUDA-rule verdict at depth 11 is "found" while this one is
"not found" is a CPU/GPU rule disagreement (a shortest ratio-valid sorting of exactly 11 moves).
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
    if m != 8:
        return None
    st, _, (e, _) = O.search_gpu_rule(list(pi), list(spi), even, float(MIN_RATE), 10, True, dedup=True, tight=True,
                                      node_limit=node_limit)
    return [case, st, e]


def main():
    scan = int(sys.argv[1]) if len(sys.argv) > 1 else 2500
    node_limit = int(sys.argv[2]) if len(sys.argv) > 2 else 50_000_000
    ctx = mp.get_context("spawn")
    with ctx.Pool(os.cpu_count()) as pool:
        rows = [r for r in pool.imap(solve, [(c, node_limit) for c in range(scan)], chunksize=1) if r is not None]
    data = {"config": 2, "m": 8, "scanned": scan, "node_limit": node_limit, "min_rate": "float32(2)/float32(1.375)",
            "rule": "sorting_search.cu:321-362 (float32), full sorting, depth 10, transposition table and tight "
                    "bound = SortingSearch.java (double prune) at depth 11 for m = 8",
            "columns": ["case", "verdict at depth 10", "nodes"], "rows": rows}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "verdicts_config2_m8.json")
    with open(path, "w") as fh:
        json.dump(data, fh, separators=(",", ":"))
    vals = [r[1] for r in rows]
    print(len(rows), {v: vals.count(v) for v in set(vals)})


if __name__ == "__main__":
    main()
