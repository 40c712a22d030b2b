"""HNSW graphs built by libpaves_gpu.so's host builder (``pv_hnsw_build``).

``Hnsw`` holds the sections of a PAVES index file (levels, level-0 lists of
stride 2M+1, upper-level slabs, entry node) and computes level-0 entry points
for queries by the upper-level greedy descent the engine runs before a GPU
graph search (engine.cpp:1539-1559, ``fv_index_graph_entry``).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import _lib
from ._lib import ptr


class Hnsw:
    """builder "host": the multi-threaded insertion builder (the engine's
    construction, pv_hnsw_build); "gpu": the bulk GPU builder
    (pv_hnsw_build_gpu) from each node's `candidates` exact nearest
    neighbours (default 4M - 1), on `device`, with BF16 tensor-core scans
    when the rows are integers the BF16 path computes exactly, else FP32."""

    def __init__(self, vectors: np.ndarray, M: int = 16, ef_construction: int = 200,
                 threads: int = 0, builder: str = "host", device: int = 0,
                 candidates: int = 0):
        L = _lib.lib()
        self.vectors = np.ascontiguousarray(vectors, np.float32)
        n, d = self.vectors.shape
        err = C.create_string_buffer(256)
        if builder == "gpu":
            v = self.vectors
            integral = bool(np.all(np.abs(v) <= 256.0) and np.array_equal(v, np.rint(v)))
            prec = _lib.FV_GPU_PREC_BF16 if integral else _lib.FV_GPU_PREC_FP32
            cand = candidates or min(1023, 4 * M - 1)
            h = L.pv_hnsw_build_gpu(ptr(v), n, d, M, cand, device, prec, err, 256)
            ef_construction = cand
        elif builder == "host":
            h = L.pv_hnsw_build(ptr(self.vectors), n, d, M, ef_construction, threads, err, 256)
        else:
            raise ValueError(f"unknown builder {builder!r}")
        if not h:
            raise RuntimeError(err.value.decode())
        self.builder = builder
        try:
            m = C.c_uint32()
            lvl = C.c_int()
            entry = C.c_uint64()
            ulen = C.c_uint64()
            L.pv_hnsw_info(h, C.byref(m), C.byref(lvl), C.byref(entry), C.byref(ulen))
            self.M = int(m.value)
            self.max_level = int(lvl.value)
            self.entry_node = int(entry.value)
            self.l0 = np.zeros((n, 2 * self.M + 1), np.uint32)
            self.levels = np.zeros(n, np.uint8)
            self.upper_offs = np.zeros(n + 1, np.uint64)
            self.upper = np.zeros(max(int(ulen.value), 1), np.uint32)
            L.pv_hnsw_export(h, ptr(self.l0), ptr(self.levels), ptr(self.upper_offs),
                             ptr(self.upper))
            self.upper = self.upper[:int(ulen.value)]
        finally:
            L.pv_hnsw_free(h)
        self.ef_construction = ef_construction

    @property
    def l0_stride(self) -> int:
        return 2 * self.M + 1

    def entries(self, queries: np.ndarray, threads: int = 0) -> np.ndarray:
        L = _lib.lib()
        q = np.ascontiguousarray(queries, np.float32)
        out = np.zeros(q.shape[0], np.uint32)
        up = self.upper if self.upper.size else np.zeros(1, np.uint32)
        rc = L.pv_hnsw_entries(ptr(self.vectors), self.vectors.shape[1], ptr(self.upper_offs),
                               ptr(up), self.M, self.max_level, self.entry_node, ptr(q),
                               q.shape[0], ptr(out), threads)
        if rc != 0:
            raise RuntimeError("pv_hnsw_entries failed")
        return out

    def write(self, path: str, cols: np.ndarray, tids: Optional[np.ndarray] = None) -> None:
        """Writes a complete PAVES index file (rows, columns, postings, graph)."""
        from .indexfile import write_index
        write_index(path, self.vectors, cols, self.M, self.ef_construction, self.levels,
                    self.l0, self.upper_offs, self.upper, self.max_level, self.entry_node,
                    tids=tids)


def build_or_load(vectors: np.ndarray, cache: Optional[str], M: int = 16,
                  ef_construction: int = 200, builder: str = "host", device: int = 0) -> Hnsw:
    """Builds a graph, or reloads the sections saved at `cache` (npz) when
    they were built from identical rows and parameters."""
    import hashlib
    key = hashlib.sha256(np.ascontiguousarray(vectors[:: max(1, len(vectors) // 4096)])
                         .tobytes()).hexdigest()[:16] + f"_{len(vectors)}_{M}_{ef_construction}_{builder}"
    if cache and os.path.exists(cache):
        z = np.load(cache)
        if str(z["key"]) == key:
            h = Hnsw.__new__(Hnsw)
            h.vectors = np.ascontiguousarray(vectors, np.float32)
            h.M, h.max_level, h.entry_node = int(z["M"]), int(z["max_level"]), int(z["entry"])
            h.l0, h.levels = z["l0"], z["levels"]
            h.upper_offs, h.upper = z["upper_offs"], z["upper"]
            h.ef_construction = ef_construction
            h.builder = builder
            return h
    h = Hnsw(vectors, M, ef_construction, builder=builder, device=device)
    if cache:
        tmp = f"{cache}.{os.getpid()}.tmp.npz"
        np.savez(tmp, key=key, M=h.M, max_level=h.max_level, entry=h.entry_node, l0=h.l0,
                 levels=h.levels, upper_offs=h.upper_offs, upper=h.upper)
        os.replace(tmp, cache)  # readers never see a partial file
    return h
