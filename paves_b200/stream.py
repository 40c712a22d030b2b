"""Uneven micro-batches through CUDA graphs with autotuned scan shapes
(libpaves_gpu.so ``pv_stream_*``).

``Stream(index, max_batch, max_k, tune_queries, tune_path)`` tunes (or
reloads the tuning of) every batch-size bucket and captures one graph per
bucket; ``run(queries, preds, k)`` serves one micro-batch with per-query
filters and k. ``Serve(index, max_batch, max_k, idle_ms)`` serves the same
batches through one persistent kernel instead (``pv_serve_*``).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import HIT_DTYPE, ptr
from .pred import Pred, concat


class Stream:
    def __init__(self, index, max_batch: int, max_k: int, tune_queries: np.ndarray,
                 tune_path: Optional[str] = None):
        self._L = _lib.lib()
        self.index = index
        self.max_batch, self.max_k = int(max_batch), int(max_k)
        tq = np.ascontiguousarray(tune_queries, np.float32)
        err = C.create_string_buffer(512)
        h = self._L.pv_stream_create(index.handle, self.max_batch, self.max_k, ptr(tq),
                                     tq.shape[0], tune_path.encode() if tune_path else None,
                                     err, len(err))
        if not h:
            raise RuntimeError(err.value.decode())
        self._h = h

    def run(self, queries: np.ndarray, preds: Sequence[Optional[Pred]], k):
        """-> (ids u64 [nq][max_k], dists f32, cnt u32 [nq], device_ms)."""
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        kk = np.ascontiguousarray(np.broadcast_to(np.asarray(k, np.uint32), (nq,)))
        bp = concat(preds, self.index.count)
        out = np.zeros(nq * self.max_k, HIT_DTYPE)
        cnt = np.zeros(nq, np.uint32)
        ms = C.c_float()
        err = C.create_string_buffer(512)
        rc = self._L.pv_stream_run(self._h, nq, ptr(q), ptr(bp.qd), ptr(bp.nodes), len(bp.nodes),
                                   ptr(bp.children), len(bp.children), ptr(bp.invals),
                                   len(bp.invals), ptr(kk), ptr(out), ptr(cnt), C.byref(ms), err,
                                   len(err))
        if rc != 0:
            raise RuntimeError(err.value.decode())
        out = out.reshape(nq, self.max_k)
        return out["node"], out["dist"], cnt, float(ms.value)

    def plans(self):
        n = self._L.pv_stream_info(self._h, -1, None, None, None, None, None, None, None)
        res = []
        for i in range(n):
            B, tb, mode, epi, ns, grow = (C.c_int(), C.c_uint32(), C.c_int(), C.c_int(), C.c_int(),
                                          C.c_int())
            ms = C.c_float()
            self._L.pv_stream_info(self._h, i, C.byref(B), C.byref(tb), C.byref(mode),
                                   C.byref(epi), C.byref(ns), C.byref(grow), C.byref(ms))
            res.append({"batch": B.value, "topb": tb.value,
                        "mode": "exact" if mode.value == _lib.PV_MODE_EXACT else "low",
                        "epi": epi.value, "stages": ns.value, "grow": grow.value,
                        "tuned_ms": round(ms.value, 4)})
        return res

    def last(self):
        u, f = C.c_int(), C.c_int()
        self._L.pv_stream_last(self._h, C.byref(u), C.byref(f))
        return {"uncertain": u.value, "fallback": f.value}

    def close(self):
        if getattr(self, "_h", None):
            self._L.pv_stream_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Serve:
    """The persistent micro-batch kernel (libpaves_gpu.so ``pv_serve_*``):
    one resident cooperative kernel consuming a queue of uneven micro-batches
    with a k and a filter per query; idle_ms without a batch lets it leave
    (the next run starts it again)."""

    def __init__(self, index, max_batch: int, max_k: int, idle_ms: int = 200):
        self._L = _lib.lib()
        self.index = index
        self.max_batch, self.max_k = int(max_batch), int(max_k)
        err = C.create_string_buffer(512)
        h = self._L.pv_serve_create(index.handle, self.max_batch, self.max_k, int(idle_ms), err,
                                    len(err))
        if not h:
            raise RuntimeError(err.value.decode())
        self._h = h

    def run(self, queries: np.ndarray, preds: Sequence[Optional[Pred]], k):
        """-> (ids u64 [nq][max_k], dists f32, cnt u32 [nq], device_ms)."""
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        kk = np.ascontiguousarray(np.broadcast_to(np.asarray(k, np.uint32), (nq,)))
        bp = concat(preds, self.index.count)
        out = np.zeros(nq * self.max_k, HIT_DTYPE)
        cnt = np.zeros(nq, np.uint32)
        ms = C.c_float()
        err = C.create_string_buffer(512)
        rc = self._L.pv_serve_run(self._h, nq, ptr(q), ptr(bp.qd), ptr(bp.nodes), len(bp.nodes),
                                  ptr(bp.children), len(bp.children), ptr(bp.invals),
                                  len(bp.invals), ptr(kk), ptr(out), ptr(cnt), C.byref(ms), err,
                                  len(err))
        if rc != 0:
            raise RuntimeError(err.value.decode())
        out = out.reshape(nq, self.max_k)
        return out["node"], out["dist"], cnt, float(ms.value)

    def status(self):
        v = [C.c_int(), C.c_int(), C.c_uint64(), C.c_int(), C.c_int(), C.c_int()]
        if self._L.pv_serve_status(self._h, *[C.byref(x) for x in v]) != 0:
            raise RuntimeError("pv_serve_status failed")
        keys = ("running", "last_exit", "batches", "graph_launch", "fallback", "uncertain")
        return {k: int(x.value) for k, x in zip(keys, v)}

    def stop(self):
        err = C.create_string_buffer(256)
        if self._L.pv_serve_stop(self._h, err, len(err)) != 0:
            raise RuntimeError(err.value.decode())

    def limits(self, idle_ms: int, barrier_ms: int, skip_cta: int = -1):
        if self._L.pv_serve_limits(self._h, idle_ms, barrier_ms, skip_cta) != 0:
            raise ValueError("pv_serve_limits: bad values")

    def close(self):
        if getattr(self, "_h", None):
            self._L.pv_serve_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
