"""Bounded run of the proof generator's sort-or-extend loop (Extensions.generate and
SortOrExtend.compute, Extensions.java:36-52, SortOrExtend.java:47-87) on the GPU frontier.

    python -m tdp1375_b200.proof_step [--levels 3] [--max-frontier 20000] [--cases out.txt]

Level 0 is the reference's three seeds: the oriented 5-cycle (0 3 1 4 2), the interleaving
pair (0 4 2)(1 5 3) and the intersecting pair (0 3 1)(2 5 4).  Each level:
  1. resolves the frontier (one canonicalisation launch, one batched search launch per
     stage, duplicates and earlier configurations searched once);
  2. writes every sorting found as a case line (spi->[moves]);
  3. extends every configuration without a sorting (a bad case) by its Type 1/2/3
     extensions into the next frontier, capped at --max-frontier configurations.
The reference recurses until no bad case is left; this driver stops after --levels levels.
"""
from __future__ import annotations

import argparse
import json
import time

from . import extend_gpu, api, casefile, extensions, frontier

SEEDS = ["(0 3 1 4 2)", "(0 4 2)(1 5 3)", "(0 3 1)(2 5 4)"]


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--levels", type=int, default=3)
    p.add_argument("--max-frontier", type=int, default=20000)
    p.add_argument("--max-n", type=int, default=63)
    p.add_argument("--cases", default="")
    p.add_argument("--table-entries", type=int, default=1 << 26)
    p.add_argument("--out", default="")
    args = p.parse_args(argv)
    api.GPUSortingSearch(1, 1, 3000 << 20, args.table_entries)
    levels = []
    found_lines = []
    try:
        f = frontier.Frontier(slot=0, max_ratio=1.375, max_depth=11)
        current = [casefile.successor(casefile.cycles_of(s)) for s in SEEDS]
        for level in range(args.levels):
            if not current:
                break
            t0 = time.perf_counter()
            f.resolve(current)
            t_resolve = time.perf_counter() - t0
            new = f.last_new
            unique_new = len(new)
            bad = [r for r in new if not r.found]
            for r in new:
                if r.found:
                    found_lines.append(casefile.format_line(r.spi, r.moves))
            t1 = time.perf_counter()
            nxt = []
            # Type 1/2 insertions of every bad case in one device launch; Type 3 on the host
            inserted, _ = extend_gpu.insertion_extensions([r.spi for r in bad]) if bad else ([], [])
            for r, ins in zip(bad, inserted):
                for ext in [e for _, e in ins] + [e for _, e in extensions.type3_extensions(r.spi)]:
                    if len(ext) <= args.max_n:
                        nxt.append(ext)
                if len(nxt) >= args.max_frontier:
                    break
            t_extend = time.perf_counter() - t1
            levels.append({"level": level, "frontier": len(current), "new_canonical": unique_new,
                           "found": sum(1 for r in new if r.found), "bad": len(bad),
                           "resolve_s": round(t_resolve, 3), "extend_s": round(t_extend, 3),
                           "configs_per_s": round(len(current) / t_resolve, 1) if t_resolve > 0 else None,
                           "stages": list(f.stage_counts)})
            f.stage_counts.clear()
            print(json.dumps(levels[-1]), flush=True)
            current = nxt[: args.max_frontier]
    finally:
        api.GPUSortingSearch.destroySlots()
    if args.cases:
        with open(args.cases, "w") as fh:
            fh.write("\n".join(found_lines) + ("\n" if found_lines else ""))
    if args.out:
        with open(args.out, "w") as fh:
            json.dump({"levels": levels, "sortings": len(found_lines)}, fh, indent=1)


if __name__ == "__main__":
    main()
