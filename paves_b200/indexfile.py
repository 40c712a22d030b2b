"""Reader and writer of the PAVES index file.

One file per index, 64-byte aligned sections after a fixed header
(engine.cpp:190-215 for ``FileHeader``, 943-1031 for the writer,
259-318 for ``fv_index_open``). The format is kept byte-for-byte so files
written by ``paves_build`` open here and files written here open in the
engine:

  header   magic "PGFAVR01", version 1, dim, count, vec_attnum, ncols,
           col_attnums[32], M, ef_construction, max_level, entry_node,
           section offsets, file_size                    (264 bytes)
  vectors  f32 [count * dim]
  tids     u64 [count]
  cols     f64 [ncols * count]   column-major, NULL = NaN
  post_vals f64 [ncols * count]  per column, values sorted (NaN last)
  post_rows u32 [ncols * count]  per column, rows in that order
  levels   u8  [count]
  l0       u32 [count * (2M+1)]  [cnt, neighbours...]
  upper_offs u64 [count + 1]     slot offsets into upper
  upper    u32 [...]             per node, per level >= 1: (M+1) slots
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass
from typing import Optional

import numpy as np

MAGIC = b"PGFAVR01"
VERSION = 1
MAX_COLS = 32
# char[8], u32 version, u32 dim, u64 count, i32 vec_attnum, u32 ncols,
# i32[32] col_attnums, u32 M, u32 efc, u32 max_level, (pad 4), u64 entry,
# 10 x u64 offsets / size
_HDR = struct.Struct("<8sIIQiI32iIII4xQ" + "Q" * 10)
assert _HDR.size == 264


def _align64(x: int) -> int:
    return (x + 63) & ~63


@dataclass
class IndexFile:
    path: str
    dim: int
    count: int
    vec_attnum: int
    ncols: int
    col_attnums: tuple
    M: int
    ef_construction: int
    max_level: int
    entry_node: int
    vectors: np.ndarray
    tids: np.ndarray
    cols: np.ndarray
    post_vals: np.ndarray
    post_rows: np.ndarray
    levels: np.ndarray
    l0: np.ndarray        # [count, 2M+1]
    upper_offs: np.ndarray
    upper: np.ndarray

    @property
    def l0_stride(self) -> int:
        return 2 * self.M + 1


def read_index(path: str) -> IndexFile:
    size = os.path.getsize(path)
    mm = np.memmap(path, np.uint8, "r")
    if size < _HDR.size:
        raise ValueError(f"bad index file {path}")
    h = _HDR.unpack(bytes(mm[:_HDR.size]))
    (magic, version, dim, count, vec_attnum, ncols), rest = h[:6], h[6:]
    col_attnums = tuple(rest[:32])
    M, efc, max_level, entry = rest[32:36]
    offs = rest[36:]
    (off_vec, off_tids, off_cols, off_pvals, off_prows, off_levels, off_l0, off_uoffs,
     off_upper, file_size) = offs
    if magic != MAGIC or version != VERSION or file_size != size:
        raise ValueError(f"index file {path}: bad magic/version/size")

    def view(off, dtype, n):
        return np.frombuffer(mm, dtype=dtype, count=n, offset=off)

    stride = 2 * M + 1
    uoffs = view(off_uoffs, np.uint64, count + 1)
    return IndexFile(
        path, dim, count, vec_attnum, ncols, col_attnums, M, efc, max_level, entry,
        view(off_vec, np.float32, count * dim).reshape(count, dim),
        view(off_tids, np.uint64, count),
        view(off_cols, np.float64, ncols * count).reshape(ncols, count),
        view(off_pvals, np.float64, ncols * count).reshape(ncols, count),
        view(off_prows, np.uint32, ncols * count).reshape(ncols, count),
        view(off_levels, np.uint8, count),
        view(off_l0, np.uint32, count * stride).reshape(count, stride),
        uoffs,
        view(off_upper, np.uint32, int(uoffs[-1])),
    )


def write_index(path: str, vectors: np.ndarray, cols: np.ndarray, M: int, ef_construction: int,
                levels: np.ndarray, l0: np.ndarray, upper_offs: np.ndarray, upper: np.ndarray,
                max_level: int, entry_node: int, tids: Optional[np.ndarray] = None,
                vec_attnum: int = 1, col_attnums: Optional[tuple] = None) -> None:
    """Writes a complete index file (tmp + fsync + rename, engine.cpp:987-1031)."""
    vectors = np.ascontiguousarray(vectors, np.float32)
    count, dim = vectors.shape
    cols = np.ascontiguousarray(cols, np.float64).reshape(-1, count)
    ncols = cols.shape[0]
    if tids is None:
        tids = np.arange(count, dtype=np.uint64)
    if col_attnums is None:
        col_attnums = tuple(range(2, 2 + ncols))
    # posting lists: rows by value, NaN last, ties by row (engine.cpp:921-941)
    prows = np.empty((ncols, count), np.uint32)
    pvals = np.empty((ncols, count), np.float64)
    for c in range(ncols):
        order = np.argsort(cols[c], kind="stable")
        prows[c] = order
        pvals[c] = cols[c][order]
    stride = 2 * M + 1
    assert l0.shape == (count, stride)
    off = _align64(_HDR.size)
    off_vec = off; off = _align64(off + count * dim * 4)
    off_tids = off; off = _align64(off + count * 8)
    off_cols = off; off = _align64(off + ncols * count * 8)
    off_pvals = off; off = _align64(off + ncols * count * 8)
    off_prows = off; off = _align64(off + ncols * count * 4)
    off_levels = off; off = _align64(off + count)
    off_l0 = off; off = _align64(off + count * stride * 4)
    off_uoffs = off; off = _align64(off + (count + 1) * 8)
    off_upper = off; off = _align64(off + len(upper) * 4)
    file_size = off
    attn = list(col_attnums) + [0] * (MAX_COLS - len(col_attnums))
    hdr = _HDR.pack(MAGIC, VERSION, dim, count, vec_attnum, ncols, *attn, M, ef_construction,
                    max_level, entry_node, off_vec, off_tids, off_cols, off_pvals, off_prows,
                    off_levels, off_l0, off_uoffs, off_upper, file_size)
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.truncate(file_size)
        for o, arr in ((0, np.frombuffer(hdr, np.uint8)), (off_vec, vectors),
                       (off_tids, np.asarray(tids, np.uint64)), (off_cols, cols),
                       (off_pvals, pvals), (off_prows, prows),
                       (off_levels, np.asarray(levels, np.uint8)),
                       (off_l0, np.ascontiguousarray(l0, np.uint32)),
                       (off_uoffs, np.asarray(upper_offs, np.uint64)),
                       (off_upper, np.asarray(upper, np.uint32))):
            f.seek(o)
            f.write(np.ascontiguousarray(arr).tobytes())
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)


# ---------------------------------------------------------------------------
# Stored device layout: a companion file "<index>.pvdev". The reference
# reader rejects a file whose size differs from its header's file_size
# (engine.cpp:274-290), so the device layout lives beside the index file
# instead of inside it, and the index file stays readable by the engine.
#
#   header   magic "PVDEVL01", version, precision, count, dim, kpad,
#            row_amax, SHA-256 of the index file's header and vectors
#            section (the rows the layout is converted from: a rewrite
#            with other vectors makes the companion stale, even when the
#            header is byte-identical because count, dim and M are),
#            section offsets, file size                         (128 bytes)
#   rows     bf16 / fp8 [count][kpad]   (row stride kpad * element size)
#   norms    f32 [count]
#   scales   f32 [count]                (FP8 only)
DEV_MAGIC = b"PVDEVL01"
DEV_VERSION = 2  # 1: digest of the header alone
# char[8], u32 version, u32 precision, u64 count, u32 dim, u32 kpad,
# f32 row_amax, (pad 4), 32s digest, 4 x u64 offsets / size, (pad 24)
_DEV_HDR = struct.Struct("<8sIIQIIf4x32sQQQQ24x")
assert _DEV_HDR.size == 128
PREC_FP8 = 3


@dataclass
class DeviceLayout:
    precision: int
    count: int
    dim: int
    kpad: int
    row_amax: float
    rows: np.ndarray            # u8 [count * kpad * element size]
    norms: np.ndarray           # f32 [count]
    scales: Optional[np.ndarray]  # f32 [count] (FP8)


def device_layout_path(path: str) -> str:
    return path + ".pvdev"


def _source_digest(path: str) -> bytes:
    """SHA-256 of the index file's header and its vectors section. The
    header alone does not identify the rows: node levels come from a hash
    of the row number (engine.cpp:720-729), so two indexes of the same
    count, dim and M have byte-identical headers."""
    import hashlib
    mm = np.memmap(path, np.uint8, "r")
    h = _HDR.unpack(bytes(mm[:_HDR.size]))
    dim, count, off_vec = h[2], h[3], h[42]
    end = off_vec + int(count) * int(dim) * 4
    if end > mm.size:
        raise ValueError(f"index file {path}: vectors section past the end")
    d = hashlib.sha256(memoryview(mm[:_HDR.size]))
    d.update(memoryview(mm[off_vec:end]))
    return d.digest()


def write_device_layout(path: str, lay: DeviceLayout) -> str:
    """Writes lay beside the index file `path` (tmp + fsync + rename)."""
    esz = 1 if lay.precision == PREC_FP8 else 2
    rows = np.ascontiguousarray(lay.rows, np.uint8).reshape(-1)
    if rows.size != lay.count * lay.kpad * esz or lay.norms.size != lay.count:
        raise ValueError("device layout arrays do not match count / kpad")
    if lay.precision == PREC_FP8 and (lay.scales is None or lay.scales.size != lay.count):
        raise ValueError("FP8 device layout needs one scale per row")
    off = _align64(_DEV_HDR.size)
    off_rows = off; off = _align64(off + rows.size)
    off_norms = off; off = _align64(off + lay.count * 4)
    off_scales = off if lay.precision == PREC_FP8 else 0
    if off_scales:
        off = _align64(off + lay.count * 4)
    size = off
    hdr = _DEV_HDR.pack(DEV_MAGIC, DEV_VERSION, lay.precision, lay.count, lay.dim, lay.kpad,
                        float(lay.row_amax), _source_digest(path), off_rows, off_norms,
                        off_scales, size)
    out = device_layout_path(path)
    tmp = out + ".tmp"
    with open(tmp, "wb") as f:
        f.truncate(size)
        parts = [(0, np.frombuffer(hdr, np.uint8)), (off_rows, rows),
                 (off_norms, np.ascontiguousarray(lay.norms, np.float32))]
        if off_scales:
            parts.append((off_scales, np.ascontiguousarray(lay.scales, np.float32)))
        for o, arr in parts:
            f.seek(o)
            f.write(arr.tobytes())
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, out)
    return out


def read_device_layout(path: str, precision: int) -> Optional[DeviceLayout]:
    """The stored device layout of index file `path` at `precision`, or None
    when there is none, it was written for another precision or by another
    version, or the index file was rewritten since (the digest of its
    header and vectors differs). A companion that
    claims to match but is malformed raises ValueError."""
    dp = device_layout_path(path)
    if not os.path.exists(dp) or os.path.getsize(dp) < _DEV_HDR.size:
        return None
    mm = np.memmap(dp, np.uint8, "r")
    (magic, version, prec, count, dim, kpad, amax, digest, off_rows, off_norms, off_scales,
     size) = _DEV_HDR.unpack(bytes(mm[:_DEV_HDR.size]))
    if magic != DEV_MAGIC or version != DEV_VERSION or prec != precision:
        return None
    if digest != _source_digest(path):
        return None
    if size != os.path.getsize(dp):
        raise ValueError(f"{dp}: truncated")
    esz = 1 if prec == PREC_FP8 else 2
    want = (dim + 127) & ~127 if prec == PREC_FP8 else (dim + 63) & ~63
    if kpad != want:
        raise ValueError(f"{dp}: row stride {kpad}, expected {want}")
    rows = np.frombuffer(mm, np.uint8, count * kpad * esz, off_rows)
    norms = np.frombuffer(mm, np.float32, count, off_norms)
    scales = np.frombuffer(mm, np.float32, count, off_scales) if prec == PREC_FP8 else None
    return DeviceLayout(prec, count, dim, kpad, amax, rows, norms, scales)
