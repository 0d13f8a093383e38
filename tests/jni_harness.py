"""Builds and runs tests/jni/fake_jvm: the real JNI bridge (tdp1375_b200/csrc/jni_bridge.cpp)
compiled against tests/jni/jni.h and linked with the product library, driven call by call
as GPUSortingSearch.java:30-45 would drive it."""
from __future__ import annotations

import json
import os
import struct
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "tdp1375_b200")


def build(out_dir: str) -> str:
    exe = os.path.join(out_dir, "fake_jvm")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "tests", "jni"),
           os.path.join(ROOT, "tdp1375_b200", "csrc", "jni_bridge.cpp"), os.path.join(ROOT, "tests", "jni", "fake_jvm.cpp"),
           "-L", LIBDIR, "-ltdp1375_jni", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


def float_bits(x: float) -> int:
    return struct.unpack("<I", struct.pack("<f", x))[0]


def search_line(slot, rate, max_moves, full, even, pi, spi, mismatch=False):
    n = len(pi)
    if mismatch:
        assert len(spi) == n - 1
        n = -n
    return f"search {slot} {float_bits(rate)} {max_moves} {1 if full else 0} {even} {n} " + \
        " ".join(str(v) for v in list(pi) + list(spi))


def filter_line(skip, n, cycle, triple):
    return f"filter {1 if skip else 0} {n} {len(cycle)} " + " ".join(map(str, cycle)) + f" {len(triple)} " + \
        " ".join(map(str, triple))


def run(exe: str, lines, tmp_dir: str):
    path = os.path.join(tmp_dir, "calls.txt")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    out = subprocess.run([exe, "calls", path], check=True, capture_output=True, text=True, timeout=600).stdout
    return [json.loads(line) for line in out.splitlines() if line.strip()]
