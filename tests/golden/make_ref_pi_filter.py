"""Generates tests/golden/ref_pi_filter.json with the reference's own CUDA permutation filter.

performGpuPiFilter (pi_filter.cu:157-260, compiled from the reference sources by
`make -C oracle ref` and driven by oracle/ref_harness.cu) runs on a B200 over seeded
(cycle, oriented triple) inputs for n = 4..11, with and without the 2-move check.  The
reference appends rows in an arbitrary order, so each record keeps the number of rows and
the SHA-256 of the rows sorted as byte strings (and the rows themselves for n <= 7), for the
optimised build and, when it is built (make -C oracle ref-debug), for the build whose
device code is unoptimised:

    python tests/golden/make_ref_pi_filter.py [--out PATH]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def inputs():
    """The filter inputs: (n, cycle, oriented triple) with the triple's symbols in the cycle.
    Seeded draws for n = 4..11, plus inputs whose triple runs against the cycle's own order
    (the three symbols in reverse cyclic order), where the triple condition and the
    orientation condition can exclude each other."""
    rng = np.random.Generator(np.random.PCG64(1375 + 3 * 10**6 + 777))
    out = []
    for n in range(4, 12):
        for _ in range(4 if n < 11 else 2):
            length = int(rng.integers(3, min(n, 9) + 1))
            cycle = [int(v) for v in rng.permutation(n)[:length]]
            triple = [int(v) for v in rng.choice(cycle, 3, replace=False)]
            out.append((n, cycle, triple))
    out += [(4, [1, 2, 3], [3, 2, 1]), (6, [4, 2, 5, 1], [5, 2, 4]), (7, [1, 3, 4, 2], [1, 2, 3]),
            (9, [8, 3, 5], [3, 8, 5]), (10, [1, 9, 4], [1, 4, 9]), (10, [9, 1, 3, 5, 7, 2, 0], [1, 0, 5])]
    return out


def digest(rows):
    h = hashlib.sha256()
    for r in sorted(rows):
        h.update(bytes(r))
    return h.hexdigest()


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_pi_filter.json"))
    args = p.parse_args()
    from oracle import reference_gpu as R
    records = []
    debug = R.available(debug=True)
    for n, cycle, triple in inputs():
        for skip in (False, True):
            rows = R.pi_filter(cycle, triple, n, skip)
            rec = {"n": n, "cycle": cycle, "triple": triple, "skip_2move_check": skip, "rows": len(rows),
                   "sha256_sorted": digest(rows)}
            if n <= 7:
                rec["sorted_rows"] = [list(r) for r in rows]
            if debug:
                rows_g = R.pi_filter(cycle, triple, n, skip, debug=True)
                rec["unoptimised"] = {"rows": len(rows_g), "sha256_sorted": digest(rows_g)}
                if n <= 7:
                    rec["unoptimised"]["sorted_rows"] = [list(r) for r in rows_g]
            records.append(rec)
    differs = sum(1 for r in records if "unoptimised" in r and r["unoptimised"]["rows"] < (1 << 20) and
                  r["unoptimised"]["sha256_sorted"] != r["sha256_sorted"])
    with open(args.out, "w") as fh:
        json.dump({"source": "reference pi_filter.cu:157-260 (performGpuPiFilter) on one B200, built by "
                             "oracle/Makefile (targets ref and ref-debug) and driven by oracle/ref_harness.cu",
                   "optimised_build_differs": differs, "records": records}, fh, separators=(",", ":"))
    print(len(records), "records")


if __name__ == "__main__":
    main()
