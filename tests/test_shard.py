"""Row-sharded scan on CPU: two and three gloo ranks each hold a slice of
the rows; one all-gather of their per-shard top-k and the merge must give
exactly the oracle's answer over the whole index (ids, FP32 distances,
counts, truncation). Each rank's own search is the oracle on its slice,
so what is checked here is the sharding: slicing, global row ids, the
exchange and the (distance, id) merge."""
import datetime
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class OracleShard:
    """The oracle over one slice of rows, with GpuIndex.brute_batch's
    signature and conventions (zeros past each query's count)."""

    def __init__(self, vectors, cols):
        self.v, self.c = vectors, cols

    def brute_batch(self, queries, preds, topb):
        from oracle import cpu
        from paves_b200 import pred
        bp = pred.concat(preds, self.v.shape[0])
        o_ids, _, o_d32, o_cnt, o_pass = cpu.exact_topk(self.v, self.c, queries, bp, topb)
        nq = queries.shape[0]
        ids = np.zeros((nq, topb), np.uint64)
        dists = np.zeros((nq, topb), np.float32)
        for q in range(nq):
            n = int(o_cnt[q])
            ids[q, :n] = o_ids[q, :n]
            dists[q, :n] = o_d32[q, :n]
        return ids, dists, np.asarray(o_cnt, np.uint32), (np.asarray(o_pass) > topb).astype(np.uint8)


def _workload():
    from paves_b200 import datagen, pred
    rng = np.random.default_rng(3)
    n = 3001  # not a multiple of the shard counts
    ds = datagen.make_dataset(n, 24, nq=12)
    cols = ds.cols.copy()
    cols[1, rng.choice(n, 40, replace=False)] = np.nan
    P, Cc = datagen.COL_PRICE, datagen.COL_CATEGORY
    preds = [None, pred.Cmp(P, "<", 10.0), pred.In(Cc, [3.0]), pred.Cmp(P, "<", -1.0),
             pred.And(pred.Cmp(P, ">=", 100.0), pred.Cmp(P, "<", 400.0)),
             pred.Not(pred.Cmp(P, "<", 990.0))] * 2
    return ds.vectors, cols, ds.queries, preds


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from paves_b200.shard import ShardedIndex, shard_range
    vectors, cols, queries, preds = _workload()
    lo, hi = shard_range(len(vectors), world, rank)
    si = ShardedIndex(vectors, cols, local=OracleShard(vectors[lo:hi], cols[:, lo:hi]))
    res = {}
    for topb in (1, 10, 700):
        ids, dists, cnt, trunc = si.brute_batch(queries, preds, topb)
        res.update({f"ids{topb}": ids, f"d{topb}": dists, f"c{topb}": cnt, f"t{topb}": trunc})
    np.savez(os.path.join(out, f"r{rank}.npz"), **res)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_ranges_cover_rows_once():
    from paves_b200.shard import shard_range
    for n in (0, 1, 7, 3001):
        for w in (1, 2, 3, 8):
            spans = [shard_range(n, w, r) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(h - l for l, h in spans) - min(h - l for l, h in spans) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_merge_to_the_whole_index_answer(world):
    from oracle import cpu
    from paves_b200 import pred
    vectors, cols, queries, preds = _workload()
    bp = pred.concat(preds, len(vectors))
    with tempfile.TemporaryDirectory() as td:
        mp.start_processes(_rank, args=(world, _free_port(), td), nprocs=world, join=True,
                           start_method="spawn")
        rs = [np.load(os.path.join(td, f"r{r}.npz")) for r in range(world)]
        for topb in (1, 10, 700):
            o_ids, _, o_d32, o_cnt, o_pass = cpu.exact_topk(vectors, cols, queries, bp, topb)
            for r in rs:  # every rank holds the same merged answer
                assert np.array_equal(r[f"c{topb}"], o_cnt.astype(np.uint32))
                assert np.array_equal(r[f"t{topb}"], (o_pass > topb).astype(np.uint8))
                for q in range(len(queries)):
                    n = int(o_cnt[q])
                    assert np.array_equal(r[f"ids{topb}"][q, :n], o_ids[q, :n].astype(np.uint64))
                    assert np.array_equal(r[f"d{topb}"][q, :n], o_d32[q, :n])
