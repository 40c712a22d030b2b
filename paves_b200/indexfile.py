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
