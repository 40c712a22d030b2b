"""Host-side handle of a device-resident index (wraps the C ABI).

``GpuIndex`` mirrors what the engine does around the reference backend:
``fv_index_gpu_ensure`` uploads (engine.cpp:1515-1535), and the batch calls
follow ``fv_gpu_exec_brute_batch`` / ``fv_gpu_exec_graph_batch``
(engine.cpp:1290-1339): concatenate the per-query predicates, call the
backend, return (ids, dists, counts, flags). Errors raise ``GpuError`` with
the backend's message (the reference returns -1 + errbuf).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import HIT_DTYPE, ptr
from .pred import BatchPred, Pred, concat


class GpuError(RuntimeError):
    pass


def _err():
    return C.create_string_buffer(512)


class GpuIndex:
    def __init__(self, vectors: np.ndarray, cols: Optional[np.ndarray] = None,
                 post_rows: Optional[np.ndarray] = None, l0: Optional[np.ndarray] = None,
                 precision: int = _lib.FV_GPU_PREC_FP32, device: int = -1, prepared=None):
        """prepared: an indexfile.DeviceLayout stored by an earlier upload of
        these rows at this precision; its low-precision rows, norms and
        scales are copied to the GPU instead of converted."""
        L = _lib.lib()
        self.vectors = np.ascontiguousarray(vectors, np.float32)
        self.count, self.dim = self.vectors.shape
        if cols is None:
            cols = np.zeros((0, self.count), np.float64)
        self.cols = np.ascontiguousarray(cols, np.float64)
        self.ncols = self.cols.shape[0]
        if post_rows is None:
            from .datagen import posting_rows
            post_rows = posting_rows(self.cols) if self.ncols else np.zeros((0, self.count),
                                                                             np.uint32)
        self.post_rows = np.ascontiguousarray(post_rows, np.uint32)
        l0_stride = 0
        if l0 is not None:
            l0 = np.ascontiguousarray(l0, np.uint32)
            l0_stride = l0.shape[1]
        err = _err()
        if prepared is not None:
            if (prepared.precision != precision or prepared.count != self.count
                    or prepared.dim != self.dim):
                raise GpuError("stored device layout does not match the rows / precision")
            rows = np.ascontiguousarray(prepared.rows)
            norms = np.ascontiguousarray(prepared.norms, np.float32)
            scales = (None if prepared.scales is None
                      else np.ascontiguousarray(prepared.scales, np.float32))
            h = L.pv_index_upload_prepared(
                ptr(self.vectors), ptr(self.cols) if self.ncols else None,
                ptr(self.post_rows) if self.ncols else None, ptr(l0) if l0 is not None else None,
                l0_stride, self.count, self.dim, self.ncols, device, precision, ptr(rows),
                ptr(norms), ptr(scales), float(prepared.row_amax), err, len(err))
        else:
            h = L.fv_gpu_index_upload(ptr(self.vectors), ptr(self.cols) if self.ncols else None,
                                      ptr(self.post_rows) if self.ncols else None,
                                      ptr(l0) if l0 is not None else None, l0_stride,
                                      self.count, self.dim, self.ncols, device, precision, err,
                                      len(err))
        if not h:
            raise GpuError(err.value.decode())
        self._h = h
        self.precision = precision
        self.has_graph = l0 is not None

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().fv_gpu_index_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device(self) -> int:
        return _lib.lib().fv_gpu_index_device(self._h)

    def export_device_layout(self):
        """This index's low-precision rows, norms and (FP8) scales as an
        indexfile.DeviceLayout (read back from the GPU)."""
        from .indexfile import DeviceLayout
        L = _lib.lib()
        parts, amax = {}, C.c_float()
        for part in (_lib.PV_PART_LOWP_ROWS, _lib.PV_PART_NORMS, _lib.PV_PART_SCALES):
            n = L.pv_index_part_bytes(self._h, part)
            if n < 0:
                continue
            buf = np.empty(n, np.uint8)
            err = _err()
            if L.pv_index_export(self._h, part, ptr(buf), n, C.byref(amax), err, len(err)) != 0:
                raise GpuError(err.value.decode())
            parts[part] = buf
        if _lib.PV_PART_LOWP_ROWS not in parts:
            raise GpuError("an FP32 index has no low-precision layout")
        esz = 1 if self.precision == _lib.FV_GPU_PREC_FP8 else 2
        scales = parts.get(_lib.PV_PART_SCALES)
        return DeviceLayout(self.precision, self.count, self.dim,
                            parts[_lib.PV_PART_LOWP_ROWS].size // (self.count * esz),
                            float(amax.value), parts[_lib.PV_PART_LOWP_ROWS],
                            parts[_lib.PV_PART_NORMS].view(np.float32),
                            None if scales is None else scales.view(np.float32))

    # ------------------------------------------------------------------
    def brute_batch_raw(self, queries: np.ndarray, bp: BatchPred, topb: int):
        L = _lib.lib()
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        out = np.zeros(nq * topb, HIT_DTYPE)
        cnt = np.zeros(nq, np.uint32)
        trunc = np.zeros(nq, np.uint8)
        err = _err()
        rc = L.fv_gpu_brute_batch(self._h, nq, ptr(q), ptr(bp.qd), ptr(bp.dedup),
                                  ptr(bp.nodes), len(bp.nodes), ptr(bp.children),
                                  len(bp.children), ptr(bp.invals), len(bp.invals),
                                  ptr(bp.spans), len(bp.spans), ptr(bp.spanoff),
                                  len(bp.spanoff), topb, ptr(out), ptr(cnt), ptr(trunc), err,
                                  len(err))
        if rc != 0:
            raise GpuError(err.value.decode())
        out = out.reshape(nq, topb)
        return out["node"], out["dist"], cnt, trunc

    def brute_batch(self, queries: np.ndarray, preds: Sequence[Optional[Pred]], topb: int):
        """Filtered top-topb per query -> (ids u64 [nq,topb], dists f32, cnt, truncated)."""
        bp = concat(preds, self.count)
        return self.brute_batch_raw(queries, bp, topb)

    def graph_batch(self, queries: np.ndarray, entries: Sequence[int],
                    preds: Sequence[Optional[Pred]], ef: int, max_visited: int = 0):
        """Filtered level-0 beam search -> (ids, dists, cnt, exhausted).
        max_visited 0 means the executor's default max(200000, 400*ef)
        (exec.c:289-290)."""
        L = _lib.lib()
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        if max_visited == 0:
            max_visited = max(200000, 400 * ef)
        bp = concat(preds, self.count, entries=entries)
        out = np.zeros(nq * ef, HIT_DTYPE)
        cnt = np.zeros(nq, np.uint32)
        exh = np.zeros(nq, np.uint8)
        err = _err()
        rc = L.fv_gpu_graph_batch(self._h, nq, ptr(q), ptr(bp.qd), ptr(bp.nodes),
                                  len(bp.nodes), ptr(bp.children), len(bp.children),
                                  ptr(bp.invals), len(bp.invals), ef, max_visited, ptr(out),
                                  ptr(cnt), ptr(exh), err, len(err))
        if rc != 0:
            raise GpuError(err.value.decode())
        out = out.reshape(nq, ef)
        return out["node"], out["dist"], cnt, exh
