"""The extend step's one-3-cycle insertions on the GPU (Extensions.java:95-141): Type 1
(configurations with open gates: insertions that touch a gate) and Type 2 (no open gate:
every insertion), one batched launch for many configurations (tdp_insertion_extensions_device).
tdp1375_b200.extensions restates the same step on signatures on the host; the two agree as
sets (tests/test_extend_gpu.py)."""
from __future__ import annotations

import ctypes
from typing import List, Sequence, Tuple

import numpy as np

from . import native


def insertion_extensions(spis: Sequence[Sequence[int]]) -> Tuple[List[List[Tuple[int, List[int]]]], List[int]]:
    """For each configuration (successor array, n <= 60): its extensions as (type, spi) in slot
    order, and its open-gate mask."""
    import torch
    lib = native.load()
    count = len(spis)
    if count == 0:
        return [], []
    max_n = max(len(s) for s in spis)
    rows = np.zeros((count, 64), np.uint8)
    ns = np.zeros(count, np.uint8)
    for r, s in enumerate(spis):
        rows[r, :len(s)] = s
        ns[r] = len(s)
    slots = int(lib.tdp_insertion_extension_slots(max_n))
    d_spi, d_n = torch.from_numpy(rows).cuda(), torch.from_numpy(ns).cuda()
    d_gates = torch.zeros(count, dtype=torch.int64, device="cuda")
    d_flags = torch.zeros(count * slots, dtype=torch.uint8, device="cuda")
    d_out = torch.zeros((count * slots, 64), dtype=torch.uint8, device="cuda")
    vp = ctypes.c_void_p
    stream = torch.cuda.current_stream()
    rc = lib.tdp_insertion_extensions_device(vp(d_spi.data_ptr()), vp(d_n.data_ptr()), count, max_n,
                                             vp(d_gates.data_ptr()), vp(d_flags.data_ptr()), vp(d_out.data_ptr()),
                                             vp(stream.cuda_stream))
    if rc != 0:
        raise RuntimeError(lib.tdp_insertion_extensions_error().decode())
    flags = d_flags.cpu().numpy().reshape(count, slots)
    out = d_out.cpu().numpy().reshape(count, slots, 64)
    gates = [int(g) & ((1 << 64) - 1) for g in d_gates.cpu().numpy()]
    result = []
    for r in range(count):
        n3 = int(ns[r]) + 3
        result.append([(int(flags[r, e]), [int(v) for v in out[r, e, :n3]]) for e in np.nonzero(flags[r])[0]])
    return result, gates
