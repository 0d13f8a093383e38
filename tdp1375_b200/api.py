"""Python mirror of the reference's Java façade ``br.unb.cic.tdp.base.GPUSortingSearch``
(GPUSortingSearch.java:19-108): a slot pool in front of the native library, the static
native methods with the same names and argument meaning, and the position -> symbol replay
of GPUSortingSearch.java:65-74.  Errors surface as ``RuntimeError`` carrying the native
message, as the JNI layer throws ``RuntimeException`` (jni_sorter.cu:16-23).
"""
from __future__ import annotations

import ctypes
import queue
from typing import Iterable, List, Sequence

import numpy as np

from . import native


def _u8(buf: Sequence[int]) -> ctypes.Array:
    arr = (ctypes.c_uint8 * max(1, len(buf)))()
    for i, v in enumerate(buf):
        arr[i] = int(v) & 0xFF
    return arr


def _raise(rc: int) -> None:
    raise RuntimeError(native.last_error() or f"tdp1375 error {rc}")


def apply_transposition(pi: bytearray, i: int, j: int, k: int) -> None:
    """Block swap of [i,j) and [j,k) in place (GPUSortingSearch.java:81-87)."""
    pi[i:k] = pi[j:k] + pi[i:j]


def positions_to_symbols(pi: Sequence[int], positions: Iterable[Sequence[int]]) -> List[List[int]]:
    """Position triples -> symbol 3-cycles by replaying block swaps (GPUSortingSearch.java:65-74)."""
    cur = bytearray(int(v) & 0xFF for v in pi)
    moves = []
    for i, j, k in positions:
        moves.append([cur[i], cur[j], cur[k]])
        apply_transposition(cur, i, j, k)
    return moves


class GPUSortingSearch:
    """Slot pool + native calls, like the Java class of the same name."""

    def __init__(self, devices_count: int, slots_per_device: int, queue_bytes_budget: int, dedup_table_size: int):
        total = devices_count * slots_per_device
        self._slots: "queue.Queue[int]" = queue.Queue(total)
        for s in range(total):
            self._slots.put(s)
        GPUSortingSearch.initSlots(total, devices_count, queue_bytes_budget, dedup_table_size)

    # ---- static natives (GPUSortingSearch.java:30-45) ---------------------------------
    @staticmethod
    def initSlots(total_slots: int, devices_count: int, queue_bytes_budget: int, dedup_table_size: int) -> None:
        rc = native.load().tdp_init_slots(total_slots, devices_count, queue_bytes_budget, dedup_table_size)
        if rc != 0:
            _raise(rc)

    @staticmethod
    def destroySlots() -> None:
        rc = native.load().tdp_destroy_slots()
        if rc != 0:
            _raise(rc)

    @staticmethod
    def searchForSortingSeq(pi: Sequence[int], spi: Sequence[int], initial_even_cycles: int, min_rate: float,
                            max_moves: int, full_sorting: bool, slot: int) -> List[List[int]]:
        """Returns the positions int[d][3] (empty when no sequence exists)."""
        n = len(pi)
        if len(spi) != n:
            raise RuntimeError("performGpuSortingSearch: inconsistent input sizes")
        out = (ctypes.c_int32 * (3 * native.MAX_DEPTH))()
        depth = ctypes.c_int32(0)
        rc = native.load().tdp_search(slot, _u8(pi), _u8(spi), n, initial_even_cycles, ctypes.c_float(min_rate),
                                      max_moves, 1 if full_sorting else 0, out, ctypes.byref(depth))
        if rc < 0 or rc == native.CANCELLED or rc == native.OVERFLOW:
            _raise(rc)
        return [[out[3 * d], out[3 * d + 1], out[3 * d + 2]] for d in range(depth.value)]

    @staticmethod
    def cancelSort(slot: int) -> None:
        rc = native.load().tdp_cancel(slot)
        if rc != 0:
            _raise(rc)

    @staticmethod
    def filterPiPermutations(cycle: Sequence[int], cycle_len: int, oriented_triple: Sequence[int], triple_len: int,
                             n: int, skip_2move_check: bool, max_rows: int = 1 << 20) -> List[bytes]:
        out = (ctypes.c_uint8 * max(1, max_rows * n))()
        hits = native.load().tdp_pi_filter(_u8(cycle), cycle_len, _u8(oriented_triple), triple_len, n,
                                           1 if skip_2move_check else 0, out, max_rows)
        if hits < 0:
            _raise(int(hits))
        rows = min(int(hits), max_rows)
        raw = bytes(out)[: rows * n]
        return [raw[r * n:(r + 1) * n] for r in range(rows)]

    # ---- instance method (GPUSortingSearch.java:47-79) --------------------------------
    def search(self, pi: Sequence[int], spi: Sequence[int], initial_even_cycles: int, min_rate: float,
               max_moves: int, full_sorting: bool) -> List[List[int]]:
        slot = self._slots.get()
        try:
            result = GPUSortingSearch.searchForSortingSeq(pi, spi, initial_even_cycles, min_rate, max_moves,
                                                          full_sorting, slot)
            if not result:
                return []
            return positions_to_symbols(pi, result)
        finally:
            self._slots.put(slot)


def make_instances(cases, max_depth: int, full_sorting: bool) -> ctypes.Array:
    """Packs (pi, spi, initial_even[, ...]) tuples into a tdp_instance array."""
    cases = list(cases)
    arr = (native.Instance * max(1, len(cases)))()
    for idx, case in enumerate(cases):
        pi, spi, even = case[0], case[1], case[2]
        inst = arr[idx]
        n = len(pi)
        inst.n = n
        inst.max_depth = max_depth
        inst.full_sorting = 1 if full_sorting else 0
        inst.initial_even_cycles = int(even)
        ctypes.memmove(inst.pi, bytes(np.asarray(pi, dtype=np.uint8)), n)
        ctypes.memmove(inst.spi, bytes(np.asarray(spi, dtype=np.uint8)), n)
    return arr


def search_batch(slot: int, instances: ctypes.Array, count: int, min_rate: float):
    """Runs tdp_search_batch; returns the Result array."""
    results = (native.Result * max(1, count))()
    rc = native.load().tdp_search_batch(slot, instances, count, ctypes.c_float(min_rate), results)
    if rc != 0:
        _raise(rc)
    return results


def last_stats(slot: int) -> native.Stats:
    st = native.Stats()
    rc = native.load().tdp_last_stats(slot, ctypes.byref(st))
    if rc != 0:
        _raise(rc)
    return st


def engine_config(slot: int) -> native.EngineConfig:
    cfg = native.EngineConfig()
    rc = native.load().tdp_get_engine_config(slot, ctypes.byref(cfg))
    if rc != 0:
        _raise(rc)
    return cfg


def set_engine_config(slot: int, cfg: native.EngineConfig) -> None:
    rc = native.load().tdp_set_engine_config(slot, ctypes.byref(cfg))
    if rc != 0:
        _raise(rc)
