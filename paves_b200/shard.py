"""Row-sharded filtered scan: an index split by rows across GPUs.

No reference counterpart: the reference engine keeps one index on one GPU
(gpu_engine.cu). The scan shards naturally by rows, so an index larger
than one GPU's memory is split into contiguous row slices; each shard
answers every query of a batch over its own rows (its own predicate
bitmaps, its own top-k), and the per-shard lists are merged by
(distance, global row id) - the order the reference sorts results by
(engine.cpp:1114-1116). Every global top-k member is in its shard's own
top-k, so the merge is exact: same rows, same FP32 distances as one index
holding every row.

Two ways to hold the shards:

* ShardedIndex - one shard per rank of a torch.distributed process group
  (one process per GPU). The exchange is ONE all-gather per batch of the
  shards' keys (nq x topb int64), counts and truncation flags (NCCL over
  NVLink between GPUs; gloo on CPU), after which every rank holds the
  merged answer.
* LocalShards - several shards in one process (e.g. the GPUs one process
  drives), merged on the host with no collective.

The graph search stays replicated (a per-shard graph would change what
the beam search finds).
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .index import GpuIndex
from .pred import Pred

KEY_NONE = np.iinfo(np.int64).max  # empty slot: sorts after every key


def shard_range(n: int, world: int, rank: int) -> Tuple[int, int]:
    """Rows [lo, hi) of shard `rank` of `world`: contiguous, sizes differ by
    at most one row."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad shard {rank} of {world}")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_keys(ids: np.ndarray, dists: np.ndarray, cnt: np.ndarray, row0: int) -> np.ndarray:
    """One shard's results -> int64 keys (distance bits << 32 | global row),
    KEY_NONE past each query's count. Squared distances are non-negative,
    so their IEEE bits order like the values (NaN after every number)."""
    nq, topb = ids.shape
    bits = np.ascontiguousarray(dists, np.float32).view(np.uint32).astype(np.int64)
    rows = ids.astype(np.int64) + int(row0)
    if rows.size and rows.max(initial=0) >= (1 << 32):
        raise ValueError("global row ids must fit 32 bits")
    keys = (bits << 32) | rows
    keys[np.arange(topb)[None, :] >= np.asarray(cnt, np.int64)[:, None]] = KEY_NONE
    return keys


def merge_keys(keys: np.ndarray, cnts: np.ndarray, truncs: np.ndarray, topb: int):
    """Per-shard keys [shards][nq][topb] -> the global top-topb per query:
    (ids u64 [nq, topb], dists f32, cnt u32, truncated u8). A query is
    truncated when some shard was, or when the shards' matches together
    exceed topb (each shard's count is then its whole match count)."""
    s, nq, tb = keys.shape
    allk = np.sort(np.transpose(keys, (1, 0, 2)).reshape(nq, s * tb), axis=1)[:, :topb]
    total = np.asarray(cnts, np.int64).sum(axis=0)
    cnt = np.minimum(total, topb).astype(np.uint32)
    trunc = (np.asarray(truncs).astype(bool).any(axis=0) | (total > topb)).astype(np.uint8)
    valid = allk != KEY_NONE
    ids = np.where(valid, allk & 0xFFFFFFFF, 0).astype(np.uint64)
    dists = np.where(valid, (allk >> 32).astype(np.uint32), 0).astype(np.uint32).view(np.float32)
    if allk.shape[1] < topb:  # fewer slots than topb in total: pad
        pad = topb - allk.shape[1]
        ids = np.pad(ids, ((0, 0), (0, pad)))
        dists = np.pad(dists, ((0, 0), (0, pad)))
    return ids, dists, cnt, trunc


def merge_shards(results: Sequence[Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray, int]],
                 topb: int):
    """results: per shard (ids, dists, cnt, truncated, first global row)."""
    keys = np.stack([shard_keys(i, d, c, r0) for i, d, c, _, r0 in results])
    return merge_keys(keys, np.stack([c for _, _, c, _, _ in results]),
                      np.stack([t for _, _, _, t, _ in results]), topb)


class LocalShards:
    """An index split by rows into shards held by one process (each shard a
    GpuIndex, on `devices[i % len(devices)]`); batches run shard by shard
    and merge on the host."""

    def __init__(self, vectors: np.ndarray, cols: Optional[np.ndarray], nshards: int,
                 precision: int = _lib.FV_GPU_PREC_FP32, devices: Sequence[int] = (-1,)):
        self.count = vectors.shape[0]
        self.shards: List[Tuple[GpuIndex, int]] = []
        for r in range(nshards):
            lo, hi = shard_range(self.count, nshards, r)
            sub_cols = None if cols is None else np.ascontiguousarray(cols[:, lo:hi])
            gi = GpuIndex(np.ascontiguousarray(vectors[lo:hi]), sub_cols, precision=precision,
                          device=devices[r % len(devices)])
            self.shards.append((gi, lo))

    def brute_batch(self, queries: np.ndarray, preds: Sequence[Optional[Pred]], topb: int):
        res = []
        for gi, lo in self.shards:
            ids, dists, cnt, trunc = gi.brute_batch(queries, preds, topb)
            res.append((ids, dists, cnt, trunc, lo))
        return merge_shards(res, topb)

    def close(self):
        for gi, _ in self.shards:
            gi.close()
        self.shards = []


class ShardedIndex:
    """This rank's shard of an index split by rows over a process group.

    Every rank calls brute_batch with the same queries, predicates and topb
    (the call is a collective); each returns the merged global answer.
    `local` replaces the shard's own index (any object with the
    GpuIndex.brute_batch signature); by default rows [lo, hi) of `vectors`
    / `cols` are uploaded to this rank's GPU."""

    def __init__(self, vectors: np.ndarray, cols: Optional[np.ndarray] = None, *, group=None,
                 precision: int = _lib.FV_GPU_PREC_FP32, device: int = -1, local=None):
        import torch
        import torch.distributed as dist
        self._dist, self._torch, self.group = dist, torch, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.count = vectors.shape[0]
        self.lo, self.hi = shard_range(self.count, self.world, self.rank)
        if local is None:
            sub_cols = None if cols is None else np.ascontiguousarray(cols[:, self.lo:self.hi])
            local = GpuIndex(np.ascontiguousarray(vectors[self.lo:self.hi]), sub_cols,
                             precision=precision, device=device)
        self.local = local
        backend = dist.get_backend(group)
        if backend == "nccl":
            dev = torch.cuda.current_device() if device < 0 else device
            self._dev = torch.device("cuda", dev)
        else:
            self._dev = torch.device("cpu")

    def brute_batch(self, queries: np.ndarray, preds: Sequence[Optional[Pred]], topb: int):
        torch, dist = self._torch, self._dist
        ids, dists, cnt, trunc = self.local.brute_batch(queries, preds, topb)
        keys = torch.from_numpy(shard_keys(ids, dists, cnt, self.lo)).to(self._dev)
        meta = torch.from_numpy(np.stack([np.asarray(cnt, np.int64),
                                          np.asarray(trunc, np.int64)])).to(self._dev)
        all_keys = [torch.empty_like(keys) for _ in range(self.world)]
        all_meta = [torch.empty_like(meta) for _ in range(self.world)]
        dist.all_gather(all_keys, keys, group=self.group)
        dist.all_gather(all_meta, meta, group=self.group)
        k = np.stack([t.cpu().numpy() for t in all_keys])
        m = np.stack([t.cpu().numpy() for t in all_meta])
        return merge_keys(k, m[:, 0, :], m[:, 1, :], topb)

    def close(self):
        if hasattr(self.local, "close"):
            self.local.close()
