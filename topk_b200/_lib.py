"""ctypes binding of libtopk_b200.so (the C ABI declared in include/topk_b200.h).

The library is the only compute path: if it is missing, importing this module
raises, and there is no CPU fallback anywhere in the package.
"""
import ctypes as C
import os
import types

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# TOPK_B200_LIB selects another build of the same ABI (e.g. the bounds-checking one).
LIB_PATH = os.environ.get("TOPK_B200_LIB") or os.path.join(_HERE, "_lib", "libtopk_b200.so")

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_OOM = 3
ERR_TIMEOUT = 4
ERR_UNSUPPORTED = 5
ERR_STATE = 6

MAX_K = 4096
MAX_Q = 64
MAX_D = 255

DIST_CORRELATED, DIST_INDEPENDENT, DIST_ANTICORRELATED, DIST_MIXED = 0, 1, 2, 3

# topk_query_batch methods (TOPK_BATCH_* in include/topk_b200.h)
BATCH_AUTO, BATCH_LOOP, BATCH_FP32, BATCH_BF16, BATCH_LEARNED = 0, 1, 2, 3, 4
ORDER_MORTON, ORDER_VTA, ORDER_PTA, ORDER_VTA_THREADS, ORDER_SLA, ORDER_KD = 0, 1, 2, 3, 4, 5


class TopKError(RuntimeError):
    """A TOPK_ERR_* status from the C ABI."""

    def __init__(self, status, message):
        self.status = status
        super().__init__(f"{status_name(status)}: {message}")


_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_H = C.c_void_p

# (name, restype, argtypes) for every entry of include/topk_b200.h
SIGNATURES = [
    ("topk_create", C.c_int, [C.c_uint64, C.c_uint32, C.c_int, C.POINTER(C.c_void_p)]),
    ("topk_destroy", C.c_int, [_H]),
    ("topk_upload_colmajor", C.c_int, [_H, _f32p, C.c_uint64]),
    ("topk_skyline_layers", C.c_int, [_H, _u32p, C.POINTER(C.c_uint64)]),
    ("topk_build_lists", C.c_int, [_H]),
    ("topk_read_list", C.c_int, [_H, C.c_uint32, _u32p, _f32p]),
    ("topk_query_ta", C.c_int, [_H, C.c_uint64, C.c_uint32, _f32p, _u8p, _u64p, _f32p, C.POINTER(C.c_uint64),
                                C.POINTER(C.c_float), _u64p]),
    ("topk_upload_rowmajor", C.c_int, [_H, _f32p, C.c_uint64]),
    ("topk_download_rowmajor", C.c_int, [_H, _f32p, C.c_uint64]),
    ("topk_csv_shape", C.c_int, [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("topk_load_csv", C.c_int, [_H, C.c_char_p, C.c_uint64, _u64p]),
    ("topk_save_csv", C.c_int, [_H, C.c_char_p]),
    ("topk_binary_shape", C.c_int, [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("topk_load_binary", C.c_int, [_H, C.c_char_p]),
    ("topk_save_binary", C.c_int, [_H, C.c_char_p]),
    ("topk_generate", C.c_int, [_H, C.c_int, C.c_uint64]),
    ("topk_normalize", C.c_int, [_H, C.c_void_p, C.c_void_p]),
    ("topk_download_colmajor", C.c_int, [_H, _f32p, C.c_uint64]),
    ("topk_query", C.c_int, [_H, C.c_uint64, C.c_uint32, _f32p, _u8p, _u64p, _f32p,
                             C.POINTER(C.c_uint64), C.POINTER(C.c_float)]),
    ("topk_query_range", C.c_int, [_H, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, _f32p, _u8p, _u64p, _f32p,
                                   C.POINTER(C.c_uint64), C.POINTER(C.c_float)]),
    ("topk_query_device", C.c_int, [_H, C.c_uint64, C.c_uint32, _f32p, _u8p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]),
    ("topk_query_range_device", C.c_int, [_H, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, _f32p, _u8p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("topk_merge_lists", C.c_int, [C.c_int, C.c_void_p, C.c_uint32, C.c_uint64, _u64p, _u64p, C.c_uint64,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64), C.c_void_p]),
    ("topk_query_batch", C.c_int, [_H, C.c_uint64, _u64p, _u32p, _f32p, C.c_uint64, _u8p, C.c_uint64, _u64p, _f32p,
                                   C.c_uint64, C.c_void_p, C.c_void_p]),
    ("topk_build_partitions", C.c_int, [_H, C.c_uint32]),
    ("topk_partition_info", C.c_int, [_H, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    ("topk_query_pruned", C.c_int, [_H, C.c_uint64, C.c_uint32, _f32p, _u8p, C.c_float, _u64p, _f32p,
                                    C.POINTER(C.c_uint64), C.POINTER(C.c_float), _u64p]),
    ("topk_mlp_param_count", C.c_uint64, [C.c_uint32]),
    ("topk_mlp_grad", C.c_int, [C.c_int, C.c_uint32, _f32p, _f32p, _f32p, C.c_uint32, _f32p, C.POINTER(C.c_float)]),
    ("topk_mlp_predict", C.c_int, [C.c_int, C.c_uint32, _f32p, _f32p, C.c_uint64, _f32p]),
    ("topk_mlp_train", C.c_int, [C.c_int, C.c_uint32, _f32p, _f32p, _f32p, C.c_uint64, C.c_uint32, C.c_uint32,
                                 C.c_float, C.c_uint64, C.c_void_p]),
    ("topk_query_features", C.c_int, [_H, C.c_uint64, _u64p, _u32p, _f32p, C.c_uint64, _u8p, C.c_uint64, _f32p,
                                      C.c_void_p]),
    ("topk_set_learned_model", C.c_int, [_H, C.c_void_p, C.c_float]),
    ("topk_get_learned_model", C.c_int, [_H, C.c_void_p, C.POINTER(C.c_float)]),
    ("topk_learned_fit", C.c_int, [_H, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                   C.c_uint32, C.c_float, C.c_uint64, C.c_void_p]),
    ("topk_query_learned", C.c_int, [_H, C.c_uint64, C.c_uint32, _f32p, _u8p, _u64p, _f32p, C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_float), _u64p, C.POINTER(C.c_float)]),
    ("topk_gather_rows", C.c_int, [_H, _u64p, C.c_uint64, _f32p]),
    ("topk_count_ge", C.c_int, [_H, C.c_uint64, C.c_uint64, C.c_uint32, _f32p, _u8p, C.c_float,
                                C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("topk_set_fault_injection", C.c_int, [_H, C.c_int]),
    ("topk_set_scan_tuning", C.c_int, [_H, C.c_uint32]),
    ("topk_set_batch_method", C.c_int, [_H, C.c_int]),
    ("topk_last_batch_stats", C.c_int, [_H, C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("topk_last_batch_info", C.c_int, [_H, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    ("topk_last_batch_switched", C.c_int, [_H, C.POINTER(C.c_uint64)]),
    ("topk_last_batch_retired", C.c_int, [_H, C.POINTER(C.c_uint64)]),
    ("topk_last_batch_filter_flops", C.c_int, [_H, C.POINTER(C.c_double)]),
    ("topk_set_batch_tiles", C.c_int, [_H, C.c_uint32, C.c_uint32]),
    ("topk_build_partitions_ordered", C.c_int, [_H, C.c_uint32, C.c_int]),
    ("topk_partition_ids", C.c_int, [_H, _u32p]),
    ("topk_get_batch_tiles", C.c_int, [_H, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("topk_tune_batch", C.c_int, [_H, C.c_uint64, _u64p, _u32p, _f32p, C.c_uint64, _u8p, C.c_uint64, _f64p]),
    ("topk_query_noalloc", C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, _f32p,
                                     _u8p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("topk_last_stats", C.c_int, [_H, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    ("topk_set_wait_limit", C.c_int, [_H, C.c_uint64]),
    ("topk_shape", C.c_int, [_H, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    ("topk_last_error", C.c_char_p, []),
    ("topk_status_name", C.c_char_p, [C.c_int]),
    ("topk_version", C.c_char_p, []),
]

_V = C.c_void_p
# Lean bindings of the per-query entry points, used by the Table methods that run
# once per query: every pointer is a plain address.  The ndpointer checks above cost
# about 1.4 us per array and call; these methods pass the addresses of their own
# per-thread call buffers instead (table.py, _CallBlock), so a call converts integers
# only.
LEAN_SIGNATURES = [
    ("topk_query", C.c_int, [_H, C.c_uint64, C.c_uint32, _V, _V, _V, _V, _V, _V]),
    ("topk_query_range", C.c_int, [_H, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint32, _V, _V, _V, _V, _V, _V]),
    ("topk_query_pruned", C.c_int, [_H, C.c_uint64, C.c_uint32, _V, _V, C.c_float, _V, _V, _V, _V, _V]),
    ("topk_query_learned", C.c_int, [_H, C.c_uint64, C.c_uint32, _V, _V, _V, _V, _V, _V, _V, _V]),
]

_lib = None
_lean = None


def lean():
    """The entry points of LEAN_SIGNATURES bound with address arguments (separate
    function objects: the checked bindings of load() stay as they are)."""
    global _lean
    if _lean is None:
        L = load()
        fns = {}
        for name, res, args in LEAN_SIGNATURES:
            fn = L[name]  # a new function object, with its own argtypes
            fn.restype = res
            fn.argtypes = args
            fns[name] = fn
        _lean = types.SimpleNamespace(**fns)
    return _lean


def load():
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libtopk_b200.so not found at {LIB_PATH}: build it with `python -m topk_b200.build` "
            "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def status_name(st):
    return load().topk_status_name(st).decode()


def check(st):
    if st != OK:
        raise TopKError(st, load().topk_last_error().decode())
    return st
