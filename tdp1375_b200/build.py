"""Builds the native library ``tdp1375_b200/libtdp1375_jni.so`` for sm_100a with nvcc.

The library name matches ``System.loadLibrary("tdp1375_jni")`` of the reference
(GPUSortingSearch.java:15-17).  The JNI bridge (csrc/jni_bridge.cpp) is added when a
``jni.h`` is found (JAVA_HOME or the usual JDK include folders), the same rule as the
reference's CMake (CMakeLists.txt:29-31).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libtdp1375_jni.so")
OBJ = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-fast-math",
              "-Xcompiler", "-ffp-contract=off"]
SOURCES = ["search_engine.cu", "pi_filter.cu", "extension_filter.cu", "canonical.cu", "mlp_gemm.cu", "mlp_kernels.cu",
           "measure.cu", "insertion_extensions.cu", "capi.cu"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def find_jni_include():
    roots = [os.environ.get("JAVA_HOME", "")] + glob.glob("/usr/lib/jvm/*")
    for root in roots:
        inc = os.path.join(root, "include")
        if root and os.path.exists(os.path.join(inc, "jni.h")):
            return [inc, os.path.join(inc, "linux")]
    return None


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(HERE, "..", "include", "tdp1375.h")]
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + headers):
            continue
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    jni = find_jni_include()
    if jni:
        src = os.path.join(CSRC, "jni_bridge.cpp")
        obj = os.path.join(OBJ, "jni_bridge.o")
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-c", src, "-o", obj] + [f"-I{p}" for p in jni] + \
            ["-I/usr/local/cuda/include"]
        subprocess.run(cmd, check=True)
        objs.append(obj)
    if _stale(OUT, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
