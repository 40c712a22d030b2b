"""ctypes wrapper of the reference engine built from its own sources
(oracle/_ref/, see oracle/Makefile). Test infrastructure and CPU baseline
only.

Entry points used (engine_api.h): fv_builder_create / add_row / finish,
fv_index_open / close, fv_pred_compile / free / serialize, fv_brute_begin,
fv_hnsw_begin, fv_cursor_next / end, fv_index_graph_entry and, for the
drop-in / reference-GPU builds, fv_engine_gpu_precision,
fv_index_gpu_ensure and fv_gpu_exec_{brute,graph}_batch.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
P = C.c_void_p


class FvPredNode(C.Structure):
    pass


FvPredNode._fields_ = [("kind", C.c_int32), ("col", C.c_int32), ("op", C.c_int32),
                       ("value", C.c_double), ("nvalues", C.c_int32),
                       ("values", C.POINTER(C.c_double)), ("nchildren", C.c_int32),
                       ("children", C.POINTER(C.POINTER(FvPredNode)))]
assert C.sizeof(FvPredNode) == 56


class FvHit(C.Structure):
    _fields_ = [("node", C.c_uint64), ("dist", C.c_float)]


class FvGpuBatchPred(C.Structure):
    _fields_ = [("nodes", P), ("nnodes", C.c_int), ("children", P), ("nchildren", C.c_int),
                ("invals", P), ("ninvals", C.c_int), ("spans", P), ("nspans", C.c_int),
                ("need_eval", C.c_int), ("dedup", C.c_int)]


def _cpu_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " avx512f " in line + " "
    except OSError:
        pass
    return False


def lib_path(kind="cpu"):
    if kind == "cpu":
        name = "libpaves_ref_cpu_v4.so" if _cpu_has_avx512() else "libpaves_ref_cpu_v3.so"
    elif kind == "dropin":
        name = "libpaves_ref_dropin.so"
    elif kind == "gpu":
        name = "libpaves_ref_gpu.so"
    else:
        raise ValueError(kind)
    return os.path.join(REF_DIR, name)


def available(kind="cpu"):
    return os.path.exists(lib_path(kind))


_libs = {}


def lib(kind="cpu"):
    if kind in _libs:
        return _libs[kind]
    path = lib_path(kind)
    if not os.path.exists(path):
        raise RuntimeError(f"{path} missing: run `make -C oracle ref` where the reference "
                           "sources are present")
    L = C.CDLL(path, mode=C.RTLD_LOCAL)
    sig = {
        "fv_builder_create": (P, [C.c_int, C.c_int, P, C.c_uint64]),
        "fv_builder_add_row": (None, [P, P, C.c_uint64, P, P]),
        "fv_builder_finish": (C.c_int, [P, C.c_char_p, C.c_int32, C.c_int, C.c_int, C.c_int,
                                        C.c_char_p, C.c_size_t]),
        "fv_builder_destroy": (None, [P]),
        "fv_index_open": (P, [C.c_char_p, C.c_char_p, C.c_size_t]),
        "fv_index_close": (None, [P]),
        "fv_pred_compile": (P, [P, C.POINTER(FvPredNode)]),
        "fv_pred_free": (None, [P]),
        "fv_pred_estimate": (C.c_uint64, [P]),
        "fv_pred_serialize": (C.c_int, [P, P, P, C.c_int, P, C.c_int, P, C.c_int, P, C.c_int,
                                        P, P]),
        "fv_brute_begin": (P, [P, P, P, C.c_int]),
        "fv_hnsw_begin": (P, [P, P, P, C.c_int, C.c_uint64]),
        "fv_cursor_next": (C.c_int, [P, P, C.c_int]),
        "fv_cursor_end": (None, [P]),
        "fv_index_graph_entry": (C.c_uint32, [P, P]),
        "fv_engine_gpu_precision": (None, [C.c_int]),
        "fv_index_gpu_ensure": (C.c_int, [P, C.c_int]),
        "fv_gpu_exec_brute_batch": (C.c_int, [P, C.c_int, P, P, C.c_uint32, P, P, P]),
        "fv_gpu_exec_graph_batch": (C.c_int, [P, C.c_int, P, P, P, C.c_uint32, C.c_uint64, P,
                                              P, P]),
    }
    for name, (rt, at) in sig.items():
        f = getattr(L, name)
        f.restype, f.argtypes = rt, at
    _libs[kind] = L
    return L


def build_index(path, vectors, cols, M=16, efc=200, threads=1, kind="cpu"):
    """fv_builder_* over rows (tid = row id) -> writes the index file."""
    L = lib(kind)
    vectors = np.ascontiguousarray(vectors, np.float32)
    cols = np.ascontiguousarray(cols, np.float64)
    n, d = vectors.shape
    ncols = cols.shape[0]
    attn = (C.c_int32 * max(ncols, 1))(*range(2, 2 + ncols))
    b = L.fv_builder_create(d, ncols, attn, n)
    rowcols = np.ascontiguousarray(cols.T)
    isnull = np.isnan(rowcols).astype(np.uint8)
    vp = vectors.ctypes.data
    rp = rowcols.ctypes.data
    npp = isnull.ctypes.data
    for i in range(n):
        L.fv_builder_add_row(b, vp + i * d * 4, i, rp + i * ncols * 8 if ncols else None,
                             npp + i * ncols if ncols else None)
    err = C.create_string_buffer(256)
    rc = L.fv_builder_finish(b, path.encode(), 1, M, efc, threads, err, 256)
    L.fv_builder_destroy(b)
    if rc != 0:
        raise RuntimeError(err.value.decode())


class RefIndex:
    def __init__(self, path, kind="cpu"):
        self.L = lib(kind)
        err = C.create_string_buffer(256)
        self.h = self.L.fv_index_open(path.encode(), err, 256)
        if not self.h:
            raise RuntimeError(err.value.decode())
        self._keep = []

    def close(self):
        if self.h:
            self.L.fv_index_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- predicates: paves_b200.pred trees -> FvPredNode trees -> FvPred
    def _node(self, p, keep):
        from paves_b200.pred import And, Cmp, In, Not, Or, OPS
        n = FvPredNode()
        keep.append(n)
        if isinstance(p, Cmp):
            n.kind, n.col, n.op, n.value = 0, p.col, OPS[p.op], p.value
        elif isinstance(p, In):
            vals = (C.c_double * max(len(p.values), 1))(*p.values)
            keep.append(vals)
            n.kind, n.col, n.nvalues = 1, p.col, len(p.values)
            n.values = C.cast(vals, C.POINTER(C.c_double))
        else:
            n.kind = {And: 2, Or: 3, Not: 4}[type(p)]
            kids = [self._node(c, keep) for c in p.children]
            arr = (C.POINTER(FvPredNode) * len(kids))(*[C.pointer(k) for k in kids])
            keep.append(arr)
            n.nchildren = len(kids)
            n.children = C.cast(arr, C.POINTER(C.POINTER(FvPredNode)))
        return n

    def compile(self, p):
        if p is None:
            return None
        keep = []
        root = self._node(p, keep)
        return self.L.fv_pred_compile(self.h, C.byref(root))

    def free_pred(self, h):
        if h:
            self.L.fv_pred_free(h)

    def _drain(self, cur, want):
        out = (FvHit * want)()
        n = self.L.fv_cursor_next(cur, out, want)
        self.L.fv_cursor_end(cur)
        ids = np.array([out[i].node for i in range(n)], np.uint64)
        ds = np.array([out[i].dist for i in range(n)], np.float32)
        return ids, ds

    def brute(self, q, pred_h, k, threads=1):
        q = np.ascontiguousarray(q, np.float32)
        cur = self.L.fv_brute_begin(self.h, q.ctypes.data, pred_h, threads)
        return self._drain(cur, k)

    def hnsw(self, q, pred_h, k, ef, max_visited=0):
        q = np.ascontiguousarray(q, np.float32)
        cur = self.L.fv_hnsw_begin(self.h, q.ctypes.data, pred_h, ef, max_visited)
        return self._drain(cur, k)

    def graph_entry(self, q):
        q = np.ascontiguousarray(q, np.float32)
        return int(self.L.fv_index_graph_entry(self.h, q.ctypes.data))

    # -- the engine's GPU batch calls (kind "gpu": the reference's own CUDA
    # backend; kind "dropin": the same engine over libpaves_gpu.so)
    def serialize(self, pred_h):
        """fv_pred_serialize (engine.cpp:1168-1224) of a compiled predicate
        into owned buffers: (FvGpuBatchPred, buffers, total_rows). None =
        no filter."""
        bp = FvGpuBatchPred()
        total = C.c_uint64(0)
        if pred_h is None:
            return bp, [], None
        nodes = np.zeros(48 * 40, np.uint8)
        children = np.zeros(96, np.int32)
        invals = np.zeros(128, np.float64)
        spans = np.zeros(4096 * 12, np.uint8)
        rc = self.L.fv_pred_serialize(self.h, pred_h, nodes.ctypes.data, 48,
                                      children.ctypes.data, 96, invals.ctypes.data, 128,
                                      spans.ctypes.data, 4096, C.byref(bp), C.byref(total))
        if rc != 0:
            raise RuntimeError("fv_pred_serialize: capacity exceeded")
        return bp, [nodes, children, invals, spans], int(total.value)

    def gpu_precision(self, precision, device=-1):
        """Sets the upload precision (0 fp32, 1 sq8) and uploads."""
        self.L.fv_engine_gpu_precision(int(precision))
        if self.L.fv_index_gpu_ensure(self.h, int(device)) != 0:
            raise RuntimeError("fv_index_gpu_ensure failed")

    def gpu_brute_batch(self, queries, bps, topb):
        """fv_gpu_exec_brute_batch (engine.cpp:1290-1313): bps one
        FvGpuBatchPred per query. Returns (ids, dists, cnt, truncated)."""
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        arr = (FvGpuBatchPred * nq)(*bps)
        out = (FvHit * (nq * topb))()
        cnt = np.zeros(nq, np.uint32)
        tr = np.zeros(nq, np.uint8)
        rc = self.L.fv_gpu_exec_brute_batch(self.h, nq, q.ctypes.data, arr, topb, out,
                                             cnt.ctypes.data, tr.ctypes.data)
        if rc != 0:
            raise RuntimeError("fv_gpu_exec_brute_batch failed")
        hits = np.frombuffer(out, np.dtype({"names": ["node", "dist"], "formats": ["<u8", "<f4"],
                                            "offsets": [0, 8], "itemsize": 16}))
        hits = hits.reshape(nq, topb)
        return hits["node"].copy(), hits["dist"].copy(), cnt, tr

    def gpu_graph_batch(self, queries, entries, bps, ef, max_visited):
        """fv_gpu_exec_graph_batch (engine.cpp:1315-1339). Returns (ids,
        dists, cnt, exhausted)."""
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        ent = np.ascontiguousarray(entries, np.uint32)
        arr = (FvGpuBatchPred * nq)(*bps)
        out = (FvHit * (nq * ef))()
        cnt = np.zeros(nq, np.uint32)
        ex = np.zeros(nq, np.uint8)
        rc = self.L.fv_gpu_exec_graph_batch(self.h, nq, q.ctypes.data, ent.ctypes.data, arr, ef,
                                            max_visited, out, cnt.ctypes.data, ex.ctypes.data)
        if rc != 0:
            raise RuntimeError("fv_gpu_exec_graph_batch failed")
        hits = np.frombuffer(out, np.dtype({"names": ["node", "dist"], "formats": ["<u8", "<f4"],
                                            "offsets": [0, 8], "itemsize": 16}))
        hits = hits.reshape(nq, ef)
        return hits["node"].copy(), hits["dist"].copy(), cnt, ex
