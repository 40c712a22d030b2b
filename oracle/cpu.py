"""ctypes wrapper of oracle/libpaves_oracle.so (see paves_oracle.c).

Test infrastructure only: the checker for the GPU path and the timed
CPU baseline."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "libpaves_oracle.so")
_lib = None
P = C.c_void_p


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} missing: run `make -C oracle`")
        L = C.CDLL(LIB)
        L.pvo_exact_topk.restype = None
        L.pvo_exact_topk.argtypes = [P, C.c_uint64, C.c_int, P, C.c_int, P, P, P, P, P, C.c_int,
                                     P, P, P, P, P, C.c_int]
        L.pvo_pred_bitmap.restype = None
        L.pvo_pred_bitmap.argtypes = [P, P, P, P, C.c_uint64, C.c_int32, P, P]
        L.pvo_graph_entry.restype = C.c_uint32
        L.pvo_graph_entry.argtypes = [P, C.c_int, P, P, C.c_uint32, C.c_int, C.c_uint64, P]
        L.pvo_hnsw_search.restype = C.c_int
        L.pvo_hnsw_search.argtypes = [P, C.c_uint64, C.c_int, P, C.c_uint32, C.c_uint32, P,
                                      C.c_int, P, P, P, P, C.c_int, C.c_uint64, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None and a.size else None


def exact_topk(vectors, cols, queries, bp, k, threads=None):
    """Exact filtered top-k. bp: a paves_b200.pred.BatchPred (its per-query
    roots index bp.nodes). Returns ids u32 [nq,k], d64, d32, cnt, passing."""
    L = lib()
    vectors = np.ascontiguousarray(vectors, np.float32)
    queries = np.ascontiguousarray(queries, np.float32)
    cols = np.ascontiguousarray(cols, np.float64)
    n, d = vectors.shape
    nq = queries.shape[0]
    roots = np.ascontiguousarray(bp.qd["proot"], np.int32)
    ids = np.zeros((nq, k), np.uint32)
    d64 = np.zeros((nq, k), np.float64)
    d32 = np.zeros((nq, k), np.float32)
    cnt = np.zeros(nq, np.uint32)
    passing = np.zeros(nq, np.uint64)
    if threads is None:
        threads = os.cpu_count() or 1
    L.pvo_exact_topk(_p(vectors), n, d, _p(queries), nq, _p(roots), _p(bp.nodes),
                     _p(bp.children), _p(bp.invals), _p(cols), k, _p(ids), _p(d64), _p(d32),
                     _p(cnt), _p(passing), threads)
    return ids, d64, d32, cnt, passing


def pred_bitmap(cols, bp, q):
    L = lib()
    cols = np.ascontiguousarray(cols, np.float64)
    n = cols.shape[1]
    words = np.zeros((n + 31) // 32, np.uint32)
    npass = np.zeros(1, np.uint64)
    L.pvo_pred_bitmap(_p(bp.nodes), _p(bp.children), _p(bp.invals), _p(cols), n,
                      int(bp.qd["proot"][q]), _p(words), _p(npass))
    return words, int(npass[0])


def graph_entry(idxf, q):
    """Upper-layer greedy descent over an IndexFile (paves_b200.indexfile)."""
    L = lib()
    q = np.ascontiguousarray(q, np.float32)
    return int(L.pvo_graph_entry(idxf.vectors.ctypes.data, idxf.dim, idxf.upper_offs.ctypes.data,
                                 idxf.upper.ctypes.data if idxf.upper.size else None, idxf.M,
                                 idxf.max_level, idxf.entry_node, q.ctypes.data))


def hnsw_search(vectors, l0, entry, q, bp, qi, cols, ef, max_visited=0):
    """One filtered beam-search phase (HnswCursor::run_phase) -> (ids, dists, exhausted)."""
    L = lib()
    vectors = np.ascontiguousarray(vectors, np.float32)
    l0 = np.ascontiguousarray(l0, np.uint32)
    q = np.ascontiguousarray(q, np.float32)
    cols = np.ascontiguousarray(cols, np.float64)
    if max_visited == 0:
        max_visited = max(200000, 400 * ef)
    ids = np.zeros(ef, np.uint32)
    dd = np.zeros(ef, np.float32)
    exh = C.c_int(0)
    root = int(bp.qd["proot"][qi]) if bp is not None else -1
    n = L.pvo_hnsw_search(_p(vectors), vectors.shape[0], vectors.shape[1], _p(l0), l0.shape[1],
                          entry, _p(q), root, _p(bp.nodes) if bp else None,
                          _p(bp.children) if bp else None, _p(bp.invals) if bp else None,
                          _p(cols), ef, max_visited, _p(ids), _p(dd), C.byref(exh))
    return ids[:n], dd[:n], bool(exh.value)
