"""Request slots and the GPU worker's micro-batch loop (libpaves_gpu.so
``pv_arbiter_*``), the thread-based restatement of the reference's
background worker (extension/paves/src/worker.c) and its shared-memory
arbiter (arbiter.c).

``Arbiter.submit`` is the backend call (arbiter.h:253
``paves_arbiter_submit``): it returns ``(rc, hits, more)`` with rc 1 =
answered, 0 = not taken (no slot, capacity, worker gone or timed out; the
caller keeps the query), -1 = the worker answered ERROR.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional

import numpy as np

from . import _lib
from ._lib import (HIT_DTYPE, NODE_DTYPE, PV_ARB_EXEC_FN, PV_STRAT_GPU_BRUTE,
                   PV_STRAT_GPU_HNSW, SPAN_DTYPE, ptr)
from .pred import Pred, serialize

__all__ = ["Arbiter", "PV_STRAT_GPU_BRUTE", "PV_STRAT_GPU_HNSW"]


class Arbiter:
    def __init__(self, nslots: int = 512, batch_max: int = 256, wait_us: int = 200,
                 idle_us: int = 60):
        self._L = _lib.lib()
        self._h = self._L.pv_arbiter_create(nslots, batch_max, wait_us, idle_us)
        if not self._h:
            raise ValueError("pv_arbiter_create: bad arguments")
        self._keep = []  # arrays borrowed by attached indexes
        self._exec = None

    def attach(self, relid: int, ino: int, index=None, count: int = 0, dim: int = 0,
               tids: Optional[np.ndarray] = None, hnsw=None) -> None:
        """Registers an index (a paves_b200.index.GpuIndex, or None with an
        executor set) under relid. hnsw (paves_b200.hnsw.Hnsw) supplies the
        upper levels for graph entry points."""
        g = index.handle if index is not None else None
        if index is not None:
            count, dim = index.count, index.dim
        keep = []
        tp = None
        if tids is not None:
            tids = np.ascontiguousarray(tids, np.uint64)
            keep.append(tids)
            tp = ptr(tids)
        vec = uo = up = None
        M = level = entry = 0
        if hnsw is not None:
            keep += [hnsw.vectors, hnsw.upper_offs, hnsw.upper]
            vec, uo = ptr(hnsw.vectors), ptr(hnsw.upper_offs)
            up = ptr(hnsw.upper) if hnsw.upper.size else None
            M, level, entry = hnsw.M, hnsw.max_level, hnsw.entry_node
        rc = self._L.pv_arbiter_attach(self._h, relid, ino, g, tp, count, dim, vec, uo, up, M,
                                       level, entry)
        if rc != 0:
            raise ValueError("pv_arbiter_attach failed (duplicate relid or bad shape)")
        self._keep.append(keep)

    def set_executor(self, fn: Optional[Callable[[_lib.PvArbBatch], int]]) -> None:
        """fn(batch) -> int replaces the GPU batch calls (None restores them)."""
        if fn is None:
            self._L.pv_arbiter_set_executor(self._h, PV_ARB_EXEC_FN(), None)
            self._exec = None
            return
        cb = PV_ARB_EXEC_FN(lambda ctx, b: int(fn(b.contents)))
        self._exec = cb
        self._L.pv_arbiter_set_executor(self._h, cb, None)

    def submit(self, relid: int, ino: int, strategy: int, query: np.ndarray,
               pred: Optional[Pred] = None, want: int = 10, max_visited: int = 0,
               sel_permille: int = 1000, timeout_ms: int = 10000, spans=None, dedup=0):
        q = np.ascontiguousarray(query, np.float32)
        if pred is not None:
            s = serialize(pred)
            nodes, children, invals = s.nodes, s.children, s.invals
        else:
            nodes = np.zeros(0, NODE_DTYPE)
            children = np.zeros(0, np.int32)
            invals = np.zeros(0, np.float64)
        sp = np.ascontiguousarray(spans if spans is not None else np.zeros(0, SPAN_DTYPE),
                                  SPAN_DTYPE)
        out = np.zeros(max(want, 1), HIT_DTYPE)
        cnt = C.c_uint32()
        more = C.c_uint8()
        rc = self._L.pv_arbiter_submit(self._h, relid, ino, strategy, q.shape[0], ptr(q),
                                       ptr(nodes), len(nodes), ptr(children), len(children),
                                       ptr(invals), len(invals), ptr(sp), len(sp), 1, dedup,
                                       want, max_visited, sel_permille, ptr(out),
                                       C.byref(cnt), C.byref(more), timeout_ms)
        return rc, out[:cnt.value].copy(), int(more.value)

    def stats(self):
        b, r, i, w = C.c_uint64(), C.c_uint64(), C.c_uint32(), C.c_int()
        self._L.pv_arbiter_stats(self._h, C.byref(b), C.byref(r), C.byref(i), C.byref(w))
        return {"batches": b.value, "requests": r.value, "inflight": i.value,
                "worker": w.value}

    def feedback(self, relid: int, strategy: int):
        q = (C.c_uint32 * 5)()
        bu, bn = C.c_uint32(), C.c_uint32()
        if self._L.pv_arbiter_feedback(self._h, relid, strategy, q, C.byref(bu),
                                       C.byref(bn)) != 0:
            return None
        return {"q_us": list(q), "batch_us": bu.value, "batch_n16": bn.value}

    def kill_worker(self) -> None:
        self._L.pv_arbiter_kill_worker(self._h)

    def close(self) -> None:
        if self._h:
            self._L.pv_arbiter_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
