"""Generates tests/golden/ref_pi_filter.json with the reference's own CUDA permutation filter.

performGpuPiFilter (pi_filter.cu:157-260, compiled from the reference sources by
`make -C oracle ref` and driven by oracle/ref_harness.cu) runs on a B200 over seeded
(cycle, oriented triple) inputs for n = 4..11, with and without the 2-move check.  The
reference appends rows in an arbitrary order, so each record keeps the number of rows and
the SHA-256 of the rows sorted as byte strings (and the rows themselves for n <= 7):

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
    """The seeded filter inputs: (n, cycle, oriented triple) with the triple inside the cycle."""
    rng = np.random.Generator(np.random.PCG64(1375 + 3 * 10**6 + 777))
    out = []
    for n in range(4, 12):
        for _ in range(4 if n < 11 else 2):
            length = int(rng.integers(3, min(n, 9) + 1))
            cycle = [int(v) for v in rng.permutation(n)[:length]]
            triple = [int(v) for v in rng.choice(cycle, 3, replace=False)]
            out.append((n, cycle, triple))
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
    for n, cycle, triple in inputs():
        for skip in (False, True):
            rows = R.pi_filter(cycle, triple, n, skip)
            rec = {"n": n, "cycle": cycle, "triple": triple, "skip_2move_check": skip, "rows": len(rows),
                   "sha256_sorted": digest(rows)}
            if n <= 7:
                rec["sorted_rows"] = [list(r) for r in rows]
            records.append(rec)
    with open(args.out, "w") as fh:
        json.dump({"source": "reference pi_filter.cu:157-260 (performGpuPiFilter) on one B200, built by "
                             "oracle/Makefile (ref) and driven by oracle/ref_harness.cu",
                   "records": records}, fh, separators=(",", ":"))
    print(len(records), "records")


if __name__ == "__main__":
    main()
