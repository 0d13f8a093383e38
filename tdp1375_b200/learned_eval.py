"""Learned move ordering, end to end: generate training pairs with the plain search, train the
BF16 MLP on the tensor cores, then compare plain and learned root order on held-out
instances (same verdicts required).

    python -m tdp1375_b200.learned_eval [--pairs 1000000] [--eval 100000] [--out result.json]

Training instances: 3-permutations from the seeded generator with seeds disjoint from the
evaluation set (config-1 sizes m in 4..6 plus m in 8..10), searched in partial mode (the
proof generator's mode) at max depth 11; every found solution contributes one
(state, next move) pair per move.  Evaluation: the held-out m in 8..10 set (seed
1375 + 5*10**6 + case), partial mode, max depth 11, one batched launch per chunk.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import api, native, order_model
from .cases import MIN_RATE, three_permutation

TRAIN_SEED_BASE = 7_000_000_000  # disjoint from every benchmark seed


def training_cases(count: int, start: int = 0):
    for case in range(start, start + count):
        rng = np.random.Generator(np.random.PCG64(TRAIN_SEED_BASE + case))
        m = int(rng.integers(4, 7)) if case % 2 == 0 else int(rng.integers(8, 11))
        yield three_permutation(m, rng)


def eval_cases(count: int):
    from .cases import config_cases
    return [c[:3] for c in config_cases(5, count)]


def collect_pairs(slot: int, target_pairs: int, chunk: int = 20000, depth: int = 11):
    spis, pis, ns, tgts = [], [], [], []
    total, start = 0, 0
    while total < target_pairs:
        cases = list(training_cases(chunk, start))
        start += chunk
        res = api.search_batch(slot, api.make_instances(cases, depth, False), len(cases), float(MIN_RATE))
        s, p, n, t = order_model.solution_pairs(cases, res)
        spis.append(s), pis.append(p), ns.append(n), tgts.append(t)
        total += len(t)
    spi, pi, n, tgt = (np.concatenate(x) for x in (spis, pis, ns, tgts))
    return spi[:target_pairs], pi[:target_pairs], n[:target_pairs], tgt[:target_pairs]


def run_eval(slot: int, cases, depth: int = 11, chunk: int = 10000):
    statuses, nodes, ms = [], 0, 0.0
    for off in range(0, len(cases), chunk):
        part = cases[off:off + chunk]
        res = api.search_batch(slot, api.make_instances(part, depth, False), len(part), float(MIN_RATE))
        st = api.last_stats(slot)
        ms += st.kernel_ms
        nodes += sum(r.nodes for r in res[:len(part)])
        statuses += [r.status for r in res[:len(part)]]
    return statuses, nodes, ms


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--pairs", type=int, default=1_000_000)
    p.add_argument("--eval", type=int, default=100_000)
    p.add_argument("--epochs", type=int, default=4)
    p.add_argument("--batch", type=int, default=4096)
    p.add_argument("--lr", type=float, default=1e-3)
    p.add_argument("--table-entries", type=int, default=1 << 28)
    p.add_argument("--out", default="")
    args = p.parse_args(argv)

    api.GPUSortingSearch(1, 1, 3000 << 20, args.table_entries)
    try:
        cfg = api.engine_config(0)
        cfg.time_limit_s = 600.0
        api.set_engine_config(0, cfg)
        t0 = time.perf_counter()
        spi, pi, n, tgt = collect_pairs(0, args.pairs)
        t_pairs = time.perf_counter() - t0
        model = order_model.OrderModel()
        t0 = time.perf_counter()
        stats = order_model.train(model, spi, pi, n, tgt, epochs=args.epochs, batch=args.batch, lr=args.lr)
        t_train = time.perf_counter() - t0
        if native.load().tdp_mlp_error() != 0:
            raise RuntimeError("tensor-core wait timed out during training")
        cases = eval_cases(args.eval)
        plain_status, plain_nodes, plain_ms = run_eval(0, cases)
        model.install(0, enable=True)
        learned_status, learned_nodes, learned_ms = run_eval(0, cases)
        identical = plain_status == learned_status
        out = {
            "pairs": int(len(tgt)), "pair_generation_s": round(t_pairs, 2), "train_s": round(t_train, 2),
            "train_steps": stats.steps, "first_loss": stats.first_loss, "last_loss": stats.last_loss,
            "train_top1": stats.top1,
            "eval_cases": len(cases), "verdicts_identical": identical,
            "found": plain_status.count(native.FOUND), "not_found": plain_status.count(native.NOT_FOUND),
            "plain": {"cases_per_s": len(cases) / (plain_ms / 1e3), "nodes": plain_nodes, "kernel_ms": plain_ms},
            "learned": {"cases_per_s": len(cases) / (learned_ms / 1e3), "nodes": learned_nodes,
                        "kernel_ms": learned_ms},
        }
        out["node_ratio_plain_over_learned"] = plain_nodes / max(1, learned_nodes)
        out["speedup_learned_over_plain"] = plain_ms / max(1e-9, learned_ms)
        print(json.dumps(out), flush=True)
        if args.out:
            with open(args.out, "w") as fh:
                json.dump(out, fh, indent=1)
        if not identical:
            raise SystemExit("verdicts differ between plain and learned order")
    finally:
        api.GPUSortingSearch.destroySlots()


if __name__ == "__main__":
    main()
