"""ctypes binding of the C ABI declared in include/tdp1375.h.

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtdp1375_jni.so")

NOT_FOUND, FOUND, CANCELLED, OVERFLOW = 0, 1, 2, 3
ERR_ARGUMENT, ERR_SLOT, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_DEVICE, ERR_NOT_INITIALISED = -1, -2, -3, -4, -5, -6
MAX_N, MAX_DEPTH = 63, 15


class Instance(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint8), ("max_depth", ctypes.c_uint8), ("full_sorting", ctypes.c_uint8),
                ("reserved", ctypes.c_uint8), ("initial_even_cycles", ctypes.c_int32),
                ("pi", ctypes.c_uint8 * 64), ("spi", ctypes.c_uint8 * 64)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("depth", ctypes.c_int32), ("nodes", ctypes.c_uint64),
                ("children", ctypes.c_uint64), ("positions", ctypes.c_int32 * 45), ("reserved", ctypes.c_int32)]


class Stats(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_uint64), ("children", ctypes.c_uint64), ("dedup_probes", ctypes.c_uint64),
                ("dedup_pruned", ctypes.c_uint64), ("dedup_inserts", ctypes.c_uint64), ("dedup_full", ctypes.c_uint64),
                ("donations", ctypes.c_uint64), ("task_pops", ctypes.c_uint64), ("kernel_ms", ctypes.c_double),
                ("error", ctypes.c_int32), ("launches", ctypes.c_int32),
                ("busy_warp_cycles", ctypes.c_uint64), ("warp_cycles", ctypes.c_uint64),
                ("dedup_replaced", ctypes.c_uint64), ("table_atomics", ctypes.c_uint64),
                ("commute_skips", ctypes.c_uint64)]


class EngineConfig(ctypes.Structure):
    _fields_ = [("blocks_per_sm", ctypes.c_int32), ("poll_interval", ctypes.c_int32), ("tight_bound", ctypes.c_int32),
                ("task_capacity", ctypes.c_int32), ("time_limit_s", ctypes.c_double),
                ("sparse_enumeration", ctypes.c_int32), ("use_cuda_graph", ctypes.c_int32),
                ("warps_per_instance", ctypes.c_int32), ("table_replacement", ctypes.c_int32),
                ("commute", ctypes.c_int32), ("probe_leaves", ctypes.c_int32)]


assert ctypes.sizeof(Instance) == 136 and ctypes.sizeof(Result) == 208

u8p = ctypes.POINTER(ctypes.c_uint8)
i32p = ctypes.POINTER(ctypes.c_int32)
vp = ctypes.c_void_p

# name -> (restype, argtypes); this list is the ABI surface that the CPU test checks.
SIGNATURES = {
    "tdp_last_error": (ctypes.c_char_p, []),
    "tdp_device_count": (ctypes.c_int, []),
    "tdp_init_slots": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_int]),
    "tdp_destroy_slots": (ctypes.c_int, []),
    "tdp_search": (ctypes.c_int, [ctypes.c_int, u8p, u8p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                  ctypes.c_int, i32p, i32p]),
    "tdp_cancel": (ctypes.c_int, [ctypes.c_int]),
    "tdp_pi_filter": (ctypes.c_int64, [u8p, ctypes.c_int, u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int, u8p,
                                       ctypes.c_int64]),
    "tdp_pi_filter_last_kernel_ms": (ctypes.c_double, []),
    "tdp_search_batch": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Instance), ctypes.c_int, ctypes.c_float,
                                        ctypes.POINTER(Result)]),
    "tdp_batch_prepare": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Instance), ctypes.c_int, ctypes.c_float]),
    "tdp_batch_run": (ctypes.c_int, [ctypes.c_int]),
    "tdp_batch_results": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Result)]),
    "tdp_last_stats": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(Stats)]),
    "tdp_get_engine_config": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(EngineConfig)]),
    "tdp_set_engine_config": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(EngineConfig)]),
    # move-ordering MLP (device pointers, stream as void*)
    "tdp_mlp_gemm": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp,
                                    ctypes.c_int, ctypes.c_int, vp]),
    "tdp_mlp_features": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, vp, vp]),
    "tdp_mlp_softmax_xent": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp, vp]),
    "tdp_mlp_transpose": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp, vp]),
    "tdp_mlp_relu_backward": (ctypes.c_int, [vp, vp, ctypes.c_int64, vp]),
    "tdp_mlp_column_sums": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp, vp]),
    "tdp_mlp_adam": (ctypes.c_int, [vp, vp, vp, vp, vp, ctypes.c_int64, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_int, vp]),
    "tdp_mlp_order": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int, vp, ctypes.c_int, vp]),
    "tdp_mlp_error": (ctypes.c_int, []),
    "tdp_set_order_model": (ctypes.c_int, [ctypes.c_int] + [vp] * 8),
    "tdp_enable_order_model": (ctypes.c_int, [ctypes.c_int, ctypes.c_int]),
    "tdp_canonical": (ctypes.c_int, [vp, vp, ctypes.c_int, vp, vp, vp]),
    "tdp_canonical_device": (ctypes.c_int, [vp, vp, ctypes.c_int, vp, vp, vp, vp]),
    "tdp_extension_count": (ctypes.c_int, [ctypes.c_int]),
    "tdp_extension_filter": (ctypes.c_int64, [vp, vp, ctypes.c_int, ctypes.c_int, vp]),
    "tdp_extension_filter_device": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp]),
    "tdp_measure_atomics": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double)]),
    "tdp_measure_last_error": (ctypes.c_char_p, []),
    "tdp_insertion_extension_slots": (ctypes.c_int64, [ctypes.c_int]),
    "tdp_insertion_extensions_device": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]),
    "tdp_insertion_extensions_error": (ctypes.c_char_p, []),
    "tdp_pi_filter_noalloc": (ctypes.c_int64, [u8p, ctypes.c_int, u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                               ctypes.c_int64, vp]),
}

_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the CUDA library (once).  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"tdp1375_b200 native library missing ({path}); run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    msg = load().tdp_last_error()
    return msg.decode() if msg else ""
