"""Autotuner for the batched search engine.

The engine's tunables and what they stand for in the batched-search design:
  * ``blocks_per_sm``      resident warps per SM, i.e. how many warps share the instances
                           (8 warps per block);
  * ``poll_interval``      chunks between a busy warp's looks at the idle-warp ring, i.e.
                           the granularity at which work is split off and donated;
  * ``warps_per_instance`` grid warps per in-flight instance (0: no cap), i.e. how many
                           instances hold live table entries at once;
  * ``table_entries``      transposition-table capacity, i.e. its load for the batch;
  * ``sparse_enumeration`` 0 every triple, 1 same-cycle pairs, 2 pairs and same-cycle
                           triples.

``tune`` times every candidate on a sample of the workload (engine kernel time from
``tdp_last_stats``; verdicts must agree across candidates), keeps the fastest, and caches
the result in a JSON file keyed by workload name and GPU name.  ``apply`` installs a cached
choice on a slot.
"""
from __future__ import annotations

import itertools
import json
import os
import time
from typing import Dict, Iterable, List, Optional

from . import api

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_cache.json")

DEFAULT_SPACE = {
    "blocks_per_sm": [0, 2, 1],
    "poll_interval": [8, 16, 32, 64],
    "sparse_enumeration": [2, 1],
}


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:  # pragma: no cover - device query is informational
        return "unknown"


def _load_cache(path: str) -> Dict:
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh)
    return {}


def candidates(space: Dict[str, List[int]]) -> Iterable[Dict[str, int]]:
    keys = sorted(space)
    for values in itertools.product(*(space[k] for k in keys)):
        yield dict(zip(keys, values))


def apply(slot: int, choice: Dict[str, int]) -> None:
    cfg = api.engine_config(slot)
    for key in ("blocks_per_sm", "poll_interval", "sparse_enumeration", "warps_per_instance"):
        if key in choice:
            setattr(cfg, key, int(choice[key]))
    api.set_engine_config(slot, cfg)


def tune(workload: str, instances, count: int, min_rate: float, table_sizes: Iterable[int] = (1 << 21, 1 << 25),
         space: Optional[Dict[str, List[int]]] = None, queue_bytes: int = 3000 << 20, repeats: int = 1,
         cache_path: str = CACHE, time_limit_s: float = 60.0) -> Dict:
    """Times every candidate on `instances` (a tdp_instance array) and caches the best.

    Creates and destroys its own slot (slot 0).  Returns the chosen configuration with its
    measured kernel time.
    """
    space = space or DEFAULT_SPACE
    results = []
    reference = None
    for entries in table_sizes:
        api.GPUSortingSearch(1, 1, queue_bytes, entries)
        try:
            for cand in candidates(space):
                cfg = api.engine_config(0)
                cfg.time_limit_s = time_limit_s
                api.set_engine_config(0, cfg)
                apply(0, cand)
                best = None
                res = None
                for _ in range(repeats):
                    res = api.search_batch(0, instances, count, min_rate)
                    ms = api.last_stats(0).kernel_ms
                    best = ms if best is None else min(best, ms)
                verdicts = [res[i].status for i in range(count)]
                if reference is None:
                    reference = verdicts
                elif verdicts != reference:
                    raise RuntimeError(f"autotune: verdicts differ for {cand} / table {entries}")
                results.append(dict(cand, table_entries=entries, kernel_ms=best))
        finally:
            api.GPUSortingSearch.destroySlots()
    choice = min(results, key=lambda r: r["kernel_ms"])
    cache = _load_cache(cache_path)
    cache[f"{workload}@{_device_name()}"] = {"choice": choice, "tried": results, "when": time.time()}
    with open(cache_path, "w") as fh:
        json.dump(cache, fh, indent=1)
    return choice


def cached(workload: str, cache_path: str = CACHE) -> Optional[Dict]:
    entry = _load_cache(cache_path).get(f"{workload}@{_device_name()}")
    return entry["choice"] if entry else None
