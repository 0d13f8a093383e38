"""Canonical-form throughput: Configuration.getCanonical / hashCode for many configurations.

    python -m tdp1375_b200.canonical_eval [--count 1000000] [--steps 10] [--out result.json]

Configurations: seeded products of m disjoint 3-cycles (m uniform in 3..10, n = 9..30),
the shape of the proof generator's configurations, as 64-byte successor rows.  Reported:
configurations/s of the device kernel with inputs resident (CUDA events around
tdp_canonical_device, a 256 MB L2 flush between launches) and through the host-buffer entry
point tdp_canonical (copies and allocation included).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

from . import native


def configurations(count: int, seed: int = 1375 + 7 * 10**6):
    rng = np.random.Generator(np.random.PCG64(seed))
    spi = np.zeros((count, 64), np.uint8)
    ns = np.zeros(count, np.uint8)
    ms = rng.integers(3, 11, size=count)
    for r in range(count):
        m = int(ms[r])
        n = 3 * m
        q = rng.permutation(n)
        row = np.arange(n)
        a, b, c = q[0::3], q[1::3], q[2::3]
        row[a], row[b], row[c] = b, c, a
        spi[r, :n] = row
        ns[r] = n
    return spi, ns


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--count", type=int, default=1_000_000)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--out", default="")
    args = p.parse_args(argv)
    import torch
    lib = native.load()
    t0 = time.perf_counter()
    spi, ns = configurations(args.count)
    t_gen = time.perf_counter() - t0
    vp = ctypes.c_void_p
    d_spi, d_n = torch.from_numpy(spi).cuda(), torch.from_numpy(ns).cuda()
    d_sig = torch.zeros((args.count, 64), dtype=torch.float32, device="cuda")
    d_h = torch.zeros(args.count, dtype=torch.int32, device="cuda")
    d_v = torch.zeros(args.count, dtype=torch.int32, device="cuda")
    flush = torch.empty(64 << 20, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def launch():
        rc = lib.tdp_canonical_device(vp(d_spi.data_ptr()), vp(d_n.data_ptr()), args.count, vp(d_sig.data_ptr()),
                                      vp(d_h.data_ptr()), vp(d_v.data_ptr()), vp(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(native.last_error())

    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    total = 0.0
    for s in range(args.steps):
        flush.fill_(s)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch()
        e1.record(stream)
        torch.cuda.synchronize()
        total += e0.elapsed_time(e1)
    dev_ms = total / args.steps
    if int((d_v < 0).sum()) != 0:
        raise SystemExit("device rejected a row")

    sig = np.zeros((args.count, 64), np.float32)
    h = np.zeros(args.count, np.int32)
    v = np.zeros(args.count, np.int32)
    w0 = time.perf_counter()
    rc = lib.tdp_canonical(spi.ctypes.data_as(vp), ns.ctypes.data_as(vp), args.count, sig.ctypes.data_as(vp),
                           h.ctypes.data_as(vp), v.ctypes.data_as(vp))
    host_ms = (time.perf_counter() - w0) * 1e3
    if rc != 0:
        raise RuntimeError(native.last_error())
    same = bool(np.array_equal(h, d_h.cpu().numpy()) and np.array_equal(sig, d_sig.cpu().numpy()))
    out = {"configurations": args.count, "n_range": [int(ns.min()), int(ns.max())], "generation_s": round(t_gen, 2),
           "device_ms": dev_ms, "configs_per_s": args.count / (dev_ms / 1e3), "host_entry_ms": host_ms,
           "host_entry_configs_per_s": args.count / (host_ms / 1e3), "device_and_host_entry_agree": same,
           "l2": "flushed by a 256 MB write between launches"}
    print(json.dumps(out), flush=True)
    if args.out:
        with open(args.out, "w") as fh:
            json.dump(out, fh, indent=1)
    if not same:
        raise SystemExit("device and host entry points disagree")


if __name__ == "__main__":
    main()
