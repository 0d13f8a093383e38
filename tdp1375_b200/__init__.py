"""B200-native transposition-sequence search (the GPUSortingSearch path of tdp1375).

The product is the CUDA library ``libtdp1375_jni.so`` (C ABI in include/tdp1375.h);
this package is its Python host: a ctypes binding, a mirror of the Java façade and the
seeded instance generators used by the tests and the benchmark.
"""
from .api import GPUSortingSearch, make_instances, positions_to_symbols, search_batch, last_stats  # noqa: F401
from . import native  # noqa: F401
