"""ctypes binding of libpaves_gpu.so (the C ABI declared in include/*.h).

The library is built in-tree (``paves_b200/libpaves_gpu.so``). There is no
fallback: if the library is missing, importing a GPU entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpaves_gpu.so")

FV_CMP_LT, FV_CMP_LE, FV_CMP_EQ, FV_CMP_GE, FV_CMP_GT, FV_CMP_NE = range(6)
FV_NODE_CMP, FV_NODE_IN, FV_NODE_AND, FV_NODE_OR, FV_NODE_NOT = range(5)
FV_GPU_PREC_FP32, FV_GPU_PREC_SQ8, FV_GPU_PREC_BF16, FV_GPU_PREC_FP8 = range(4)
FV_GPU_MAX_TOPB = 4096
FV_GPU_MAX_SPANS = 4096
FV_GPU_MAX_EF = 512
FV_GPU_MAX_BATCH = 1024


class FvGpuPredNode(C.Structure):
    _fields_ = [("kind", C.c_int32), ("col", C.c_int32), ("op", C.c_int32),
                ("nchildren", C.c_int32), ("child0", C.c_int32),
                ("nvalues", C.c_int32), ("val0", C.c_int32), ("pad", C.c_int32),
                ("value", C.c_double)]


class FvGpuSpan(C.Structure):
    _fields_ = [("col", C.c_int32), ("lo", C.c_uint32), ("hi", C.c_uint32)]


class FvHit(C.Structure):
    _fields_ = [("node", C.c_uint64), ("dist", C.c_float)]


class FvGpuQueryDesc(C.Structure):
    _fields_ = [("proot", C.c_int32), ("need_eval", C.c_int32), ("span0", C.c_int32),
                ("nspans", C.c_int32), ("soff0", C.c_int32), ("entry", C.c_uint32),
                ("total", C.c_uint64)]


assert C.sizeof(FvGpuPredNode) == 40 and C.sizeof(FvGpuSpan) == 12
assert C.sizeof(FvHit) == 16 and C.sizeof(FvGpuQueryDesc) == 32

# numpy mirrors (same byte layout) for bulk construction
NODE_DTYPE = np.dtype([("kind", "<i4"), ("col", "<i4"), ("op", "<i4"), ("nchildren", "<i4"),
                       ("child0", "<i4"), ("nvalues", "<i4"), ("val0", "<i4"), ("pad", "<i4"),
                       ("value", "<f8")])
SPAN_DTYPE = np.dtype([("col", "<i4"), ("lo", "<u4"), ("hi", "<u4")])
HIT_DTYPE = np.dtype({"names": ["node", "dist"], "formats": ["<u8", "<f4"],
                      "offsets": [0, 8], "itemsize": 16})
QD_DTYPE = np.dtype([("proot", "<i4"), ("need_eval", "<i4"), ("span0", "<i4"),
                     ("nspans", "<i4"), ("soff0", "<i4"), ("entry", "<u4"), ("total", "<u8")])
assert NODE_DTYPE.itemsize == 40 and QD_DTYPE.itemsize == 32 and SPAN_DTYPE.itemsize == 12

_lib = None

P = C.c_void_p
_SIGS = {
    "fv_gpu_available": (C.c_int, []),
    "fv_gpu_index_upload": (P, [P, P, P, P, C.c_uint32, C.c_uint64, C.c_int, C.c_int, C.c_int,
                                C.c_int, C.c_char_p, C.c_size_t]),
    "fv_gpu_index_free": (None, [P]),
    "fv_gpu_index_device": (C.c_int, [P]),
    "fv_gpu_index_precision": (C.c_int, [P]),
    "fv_gpu_brute_batch": (C.c_int, [P, C.c_int, P, P, P, P, C.c_int, P, C.c_int, P, C.c_int,
                                     P, C.c_int, P, C.c_int, C.c_uint32, P, P, P, C.c_char_p,
                                     C.c_size_t]),
    "fv_gpu_graph_batch": (C.c_int, [P, C.c_int, P, P, P, C.c_int, P, C.c_int, P, C.c_int,
                                     C.c_uint32, C.c_uint64, P, P, P, C.c_char_p, C.c_size_t]),
    "fv_gpu_tile_variant_qt": (C.c_int, [C.c_int]),
    "fv_gpu_mem_probe": (C.c_int, [P, P]),
}


def exported_symbols():
    """Names the library must export: every function declared in include/*.h."""
    return list(_SIGS) + list(_EXT_SIGS)


_EXT_SIGS = {
    "pv_pred_check": (C.c_int, [C.c_int, P, P, C.c_int, P, C.c_int, P, C.c_int, C.c_int, P,
                                C.c_char_p, C.c_size_t]),
    "pv_batch_create": (P, [P, C.c_int, P, P, P, C.c_int, P, C.c_int, P, C.c_int, C.c_uint32,
                            C.c_int, C.c_char_p, C.c_size_t]),
    "pv_batch_run": (C.c_int, [P, C.c_int, P, P, C.c_char_p, C.c_size_t]),
    "pv_batch_fetch": (C.c_int, [P, P, P, P, C.c_char_p, C.c_size_t]),
    "pv_batch_free": (None, [P]),
    "pv_brute_batch_noalloc": (C.c_int, [P, C.c_int, P, C.c_uint32, P, P, C.c_char_p,
                                         C.c_size_t]),
    "pv_hnsw_build": (P, [P, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p,
                          C.c_size_t]),
    "pv_hnsw_free": (None, [P]),
    "pv_hnsw_info": (C.c_int, [P, P, P, P, P]),
    "pv_hnsw_export": (C.c_int, [P, P, P, P, P]),
    "pv_hnsw_entries": (C.c_int, [P, C.c_int, P, P, C.c_uint32, C.c_int, C.c_uint64, P, C.c_int,
                                  P, C.c_int]),
    "pv_last_kernel_ms": (C.c_float, [P]),
    "pv_last_superset": (C.c_int, [P]),
    "pv_last_launches": (C.c_int, [P]),
    "pv_last_uncertain": (C.c_int, [P]),
    "pv_graph_stats": (C.c_int, [P, P, C.c_int]),
}
PV_MODE_EXACT, PV_MODE_LOW = 0, 1


def register_ext(name, restype, argtypes):
    _EXT_SIGS[name] = (restype, argtypes)
    if _lib is not None:
        f = getattr(_lib, name)
        f.restype, f.argtypes = restype, argtypes


def lib():
    """Loads libpaves_gpu.so once; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
                "g.build()'` (or make -C paves_b200/csrc)")
        L = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
        for name, (rt, at) in list(_SIGS.items()) + list(_EXT_SIGS.items()):
            f = getattr(L, name)
            f.restype, f.argtypes = rt, at
        _lib = L
    return _lib


def ptr(a):
    """Address of a contiguous numpy array (None for None / empty)."""
    if a is None:
        return None
    return a.ctypes.data if a.size else None


class PvArbBatch(C.Structure):
    _fields_ = [("g", P), ("strategy", C.c_int), ("nq", C.c_int), ("dim", C.c_int),
                ("queries", P), ("qd", P), ("dedup", P), ("nodes", P), ("nnodes", C.c_int),
                ("children", P), ("nchildren", C.c_int), ("invals", P), ("ninvals", C.c_int),
                ("spans", P), ("nspans", C.c_int), ("spanoff", P), ("nspanoff", C.c_int),
                ("want", C.c_uint32), ("max_visited", C.c_uint64), ("out", P), ("out_cnt", P),
                ("flags", P)]


PV_ARB_EXEC_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(PvArbBatch))
PV_STRAT_GPU_BRUTE, PV_STRAT_GPU_HNSW = 3, 4
PV_ARB_MAX_DIM, PV_ARB_MAX_NODES, PV_ARB_MAX_RESULTS = 2000, 48, 1024

_EXT_SIGS.update({
    "pv_arbiter_create": (P, [C.c_int, C.c_int, C.c_int, C.c_int]),
    "pv_arbiter_attach": (C.c_int, [P, C.c_uint32, C.c_uint64, P, P, C.c_uint64, C.c_int, P, P,
                                    P, C.c_uint32, C.c_int, C.c_uint64]),
    "pv_arbiter_set_executor": (None, [P, PV_ARB_EXEC_FN, P]),
    "pv_arbiter_submit": (C.c_int, [P, C.c_uint32, C.c_uint64, C.c_int, C.c_int, P, P, C.c_int,
                                    P, C.c_int, P, C.c_int, P, C.c_int, C.c_int, C.c_int,
                                    C.c_uint32, C.c_uint64, C.c_int, P, P, P, C.c_int]),
    "pv_arbiter_stats": (C.c_int, [P, P, P, P, P]),
    "pv_arbiter_feedback": (C.c_int, [P, C.c_uint32, C.c_int, P, P, P]),
    "pv_arbiter_kill_worker": (None, [P]),
    "pv_arbiter_destroy": (None, [P]),
})

PV_MLP_IN, PV_MLP_HIDDEN, PV_MLP_OUT = 12, 64, 5
PV_MLP_NPARAMS = 12 * 64 + 64 + 64 * 64 + 64 + 64 * 5 + 5
_EXT_SIGS.update({
    "pv_router_create": (P, [C.c_int, P, C.c_int, C.c_int, C.c_char_p, C.c_size_t]),
    "pv_router_free": (None, [P]),
    "pv_router_set_params": (C.c_int, [P, P, P, P, C.c_char_p, C.c_size_t]),
    "pv_router_get_params": (C.c_int, [P, P, P, P]),
    "pv_router_features": (C.c_int, [P, P, C.c_int, P, P, P, C.c_int, P, C.c_int, P, C.c_int, P,
                                     P, C.c_char_p, C.c_size_t]),
    "pv_router_forward": (C.c_int, [P, C.c_int, P, P, C.c_char_p, C.c_size_t]),
    "pv_router_grad": (C.c_int, [P, C.c_int, P, P, P, P, P, C.c_char_p, C.c_size_t]),
    "pv_router_train": (C.c_int, [P, C.c_int, P, P, P, C.c_int, C.c_int, C.c_float, C.c_uint64,
                                  P, C.c_char_p, C.c_size_t]),
})
_EXT_SIGS["pv_routed_batch"] = (C.c_int, [P, P, C.c_int, P, P, P, C.c_int, P, C.c_int, P, C.c_int,
                                          P, C.c_uint32, P, C.c_float, C.c_int, P, P, P, P, P,
                                          C.c_char_p, C.c_size_t])

PV_STREAM_MAX_K = 256
_EXT_SIGS.update({
    "pv_stream_create": (P, [P, C.c_int, C.c_uint32, P, C.c_int, C.c_char_p, C.c_char_p,
                             C.c_size_t]),
    "pv_stream_run": (C.c_int, [P, C.c_int, P, P, P, C.c_int, P, C.c_int, P, C.c_int, P, P, P, P,
                                C.c_char_p, C.c_size_t]),
    "pv_stream_info": (C.c_int, [P, C.c_int, P, P, P, P, P, P, P]),
    "pv_stream_last": (C.c_int, [P, P, P]),
    "pv_stream_free": (None, [P]),
})
_EXT_SIGS["pv_last_sparse"] = (C.c_int, [P])
_EXT_SIGS["pv_index_part_bytes"] = (C.c_int64, [P, C.c_int])
_EXT_SIGS["pv_index_export"] = (C.c_int, [P, C.c_int, P, C.c_uint64, P, C.c_char_p, C.c_size_t])
_EXT_SIGS["pv_index_upload_prepared"] = (P, [P, P, P, P, C.c_uint32, C.c_uint64, C.c_int, C.c_int,
                                             C.c_int, C.c_int, P, P, P, C.c_float, C.c_char_p,
                                             C.c_size_t])
PV_PART_LOWP_ROWS, PV_PART_NORMS, PV_PART_SCALES = 1, 2, 3
_EXT_SIGS["pv_tc_shape"] = (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int])
_EXT_SIGS["pv_tc_wide_superset"] = (C.c_int, [P, C.c_int])
_EXT_SIGS["pv_exact_tc"] = (C.c_int, [P, C.c_int])
_EXT_SIGS["pv_last_exact_tc"] = (C.c_int, [P])
_EXT_SIGS["pv_hnsw_build_gpu"] = (P, [P, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_char_p, C.c_size_t])
PV_SERVE_MAX_K = 256
_EXT_SIGS.update({
    "pv_serve_create": (P, [P, C.c_int, C.c_uint32, C.c_uint32, C.c_char_p, C.c_size_t]),
    "pv_serve_run": (C.c_int, [P, C.c_int, P, P, P, C.c_int, P, C.c_int, P, C.c_int, P, P, P, P,
                               C.c_char_p, C.c_size_t]),
    "pv_serve_status": (C.c_int, [P, P, P, P, P, P, P]),
    "pv_serve_stop": (C.c_int, [P, C.c_char_p, C.c_size_t]),
    "pv_serve_limits": (C.c_int, [P, C.c_uint32, C.c_uint32, C.c_int]),
    "pv_serve_free": (None, [P]),
})
_EXT_SIGS["pv_tc_timeout"] = (C.c_int, [P, C.c_uint64])
_EXT_SIGS["pv_filter_bound"] = (C.c_int, [P, P, C.c_int, P, C.c_int, P, C.c_int, P, C.c_char_p,
                                          C.c_size_t])
