"""Extension enumeration throughput: every one-3-cycle extension of many base configurations
through the batched permutation filter.

    python -m tdp1375_b200.extension_eval [--bases 1000] [--steps 20] [--out result.json]

Bases: ``cases.extension_bases`` (m = 6 disjoint 3-cycles, n = 18, pi the identity).  Each
base has tdp_extension_count(18) = 2*C(18,3) + 2*C(21,3) = 4292 candidates.  Reported: the
hit count, candidates/s and bases/s of the device kernel with inputs resident (CUDA events
around ``tdp_extension_filter_device``), and the same through the host-buffer entry point
``tdp_extension_filter`` (copies and allocation included).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

from . import native
from .cases import extension_bases


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--bases", type=int, default=1000)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--out", default="")
    args = p.parse_args(argv)
    import torch
    lib = native.load()
    pi, spi, n = extension_bases(args.bases)
    per = lib.tdp_extension_count(n)
    total = per * args.bases

    keep_host = np.zeros(total, np.uint8)
    vp = ctypes.c_void_p
    hits = lib.tdp_extension_filter(spi.ctypes.data_as(vp), pi.ctypes.data_as(vp), n, args.bases,
                                    keep_host.ctypes.data_as(vp))
    if hits < 0:
        raise RuntimeError(native.last_error())

    d_spi, d_pi = torch.from_numpy(spi).cuda(), torch.from_numpy(pi).cuda()
    d_keep = torch.zeros(total, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def launch():
        rc = lib.tdp_extension_filter_device(vp(d_spi.data_ptr()), vp(d_pi.data_ptr()), n, args.bases,
                                             vp(d_keep.data_ptr()), vp(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(native.last_error())

    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        launch()
    t1.record(stream)
    torch.cuda.synchronize()
    dev_ms = t0.elapsed_time(t1) / args.steps
    same = bool(np.array_equal(d_keep.cpu().numpy(), keep_host))

    for _ in range(args.warmup):
        lib.tdp_extension_filter(spi.ctypes.data_as(vp), pi.ctypes.data_as(vp), n, args.bases,
                                 keep_host.ctypes.data_as(vp))
    w0 = time.perf_counter()
    for _ in range(args.steps):
        lib.tdp_extension_filter(spi.ctypes.data_as(vp), pi.ctypes.data_as(vp), n, args.bases,
                                 keep_host.ctypes.data_as(vp))
    host_ms = (time.perf_counter() - w0) * 1e3 / args.steps

    out = {
        "bases": args.bases, "n": n, "candidates_per_base": per, "candidates": total, "hits": int(hits),
        "hits_per_base_mean": hits / args.bases, "device_and_host_entry_agree": same,
        "device_ms": dev_ms, "candidates_per_s": total / (dev_ms / 1e3), "bases_per_s": args.bases / (dev_ms / 1e3),
        "host_entry_ms": host_ms, "host_entry_bases_per_s": args.bases / (host_ms / 1e3),
    }
    print(json.dumps(out), flush=True)
    if args.out:
        with open(args.out, "w") as fh:
            json.dump(out, fh, indent=1)
    if not same:
        raise SystemExit("device and host entry points disagree")


if __name__ == "__main__":
    main()
