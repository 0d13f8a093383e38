"""Generates the golden fixtures under tests/golden/ from the reference checkout.

Run from the repository root with the reference mounted:
    python tests/golden/make_golden.py /path/to/reference

Outputs (small JSON files, committed):
  cases_comb.json      src/main/resources/cases/cases-comb.txt       (ratio 1.375, depth <= 11)
  cases_3_2.json       src/main/resources/cases/cases-3,2.txt        (ratio 1.5)
  cases_7cycle.json    src/main/resources/cases/cases-oriented-7cycle.txt
Each record: {"spi": one-line spi (n bytes), "pi": pi array, "moves": [[a,b,c], ...] symbol
3-cycles, "line": the case line as written in the file}.  pi is the identity array except for the oriented 7-cycle file, whose left side is
pi itself with spi = (0 3 4 1 5 2 6) (Silvaetal.java:151-165).
The text format is the one parsed by AbstractSbtAlgorithm.java:166-179: "cycles->[moves]".
"""
from __future__ import annotations

import json
import os
import re
import sys

FILES = {
    "cases_comb.json": "src/main/resources/cases/cases-comb.txt",
    "cases_3_2.json": "src/main/resources/cases/cases-3,2.txt",
    "cases_7cycle.json": "src/main/resources/cases/cases-oriented-7cycle.txt",
}


def parse_cycles(text: str):
    return [[int(t) for t in grp.replace(",", " ").split()] for grp in re.findall(r"\(([^()]*)\)", text)]


def one_line(cycles):
    symbols = sorted(s for c in cycles for s in c)
    n = len(symbols)
    if symbols != list(range(n)):
        raise ValueError("cycles do not cover 0..n-1")
    spi = list(range(n))
    for c in cycles:
        for idx, s in enumerate(c):
            spi[s] = c[(idx + 1) % len(c)]
    return spi


def main(ref: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    for out, rel in FILES.items():
        records = []
        with open(os.path.join(ref, rel)) as fh:
            for line in fh:
                line = line.strip()
                if not line:
                    continue
                left, right = line.split("->")
                if out == "cases_7cycle.json":
                    pi = parse_cycles(left)[0]
                    spi = one_line([[0, 3, 4, 1, 5, 2, 6]])
                else:
                    spi = one_line(parse_cycles(left))
                    pi = list(range(len(spi)))
                records.append({"spi": spi, "pi": pi, "moves": parse_cycles(right), "line": line})
        with open(os.path.join(here, out), "w") as fh:
            json.dump({"source": rel, "records": records}, fh, separators=(",", ":"))
        print(out, len(records))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
