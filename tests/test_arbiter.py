"""Worker micro-batch loop (pv_arbiter_*) on the host: batching, predicate
concatenation, graph ordering and entry points, prefix/tid/more semantics,
errors, reclaim after a dead or stuck worker. The GPU batch is replaced by
an executor that answers from the oracle, so no device is involved
(worker.c:149-598 and arbiter.c:108-269 are the behaviour followed)."""
import ctypes
import threading
import time

import numpy as np
import pytest

from oracle import cpu
from paves_b200 import datagen, pred
from paves_b200._lib import HIT_DTYPE, NODE_DTYPE, QD_DTYPE, PvArbBatch
from paves_b200.arbiter import PV_STRAT_GPU_BRUTE, PV_STRAT_GPU_HNSW, Arbiter
from paves_b200.hnsw import Hnsw

N, D = 3000, 16


@pytest.fixture(scope="module")
def ds():
    return datagen.make_dataset(N, D, nq=96)


def _arr(p, dtype, n):
    if n == 0 or not p:
        return np.zeros(0, dtype)
    return np.frombuffer((ctypes.c_ubyte * (n * dtype.itemsize)).from_address(p), dtype).copy()


def _out(b):
    n = b.nq * b.want
    buf = (ctypes.c_ubyte * (n * HIT_DTYPE.itemsize)).from_address(b.out)
    return np.frombuffer(buf, HIT_DTYPE).reshape(b.nq, b.want)


def _view(b: PvArbBatch):
    """numpy copies of a batch handed to the executor."""
    nq = b.nq
    q = _arr(b.queries, np.dtype(np.float32), nq * b.dim).reshape(nq, b.dim)
    qd = _arr(b.qd, QD_DTYPE, nq)
    nodes = _arr(b.nodes, NODE_DTYPE, b.nnodes)
    children = _arr(b.children, np.dtype(np.int32), b.nchildren)
    invals = _arr(b.invals, np.dtype(np.float64), b.ninvals)
    return q, qd, nodes, children, invals


class OracleExec:
    """Executor answering each batch with the oracle's exact filtered top-k
    at the batch's want (the result a correct GPU batch gives)."""

    def __init__(self, ds, cnt_extra=0, flag=0, rc=0, bad_id_at=None, delay=0.0):
        self.ds, self.cnt_extra, self.flag, self.rc = ds, cnt_extra, flag, rc
        self.bad_id_at, self.delay = bad_id_at, delay
        self.batches = []
        self.gate = None

    def __call__(self, b: PvArbBatch) -> int:
        if self.gate is not None:
            self.gate.wait(5)
        if self.delay:
            time.sleep(self.delay)
        q, qd, nodes, children, invals = _view(b)
        self.batches.append({"nq": b.nq, "strategy": b.strategy, "want": b.want,
                             "entries": qd["entry"].copy(), "mv": b.max_visited,
                             "q": q.copy()})
        if self.rc < 0:
            return self.rc
        bp = pred.BatchPred(qd, nodes, children, invals, None, None, None)
        ids, _, d32, cnt, _ = cpu.exact_topk(self.ds.vectors, self.ds.cols, q, bp, b.want,
                                             threads=2)
        out = _out(b)
        out["node"] = ids
        out["dist"] = d32
        if self.bad_id_at is not None:
            out["node"][:, self.bad_id_at] = N + 5
        oc = np.frombuffer((ctypes.c_uint32 * b.nq).from_address(b.out_cnt), np.uint32)
        fl = np.frombuffer((ctypes.c_uint8 * b.nq).from_address(b.flags), np.uint8)
        oc[:] = cnt + self.cnt_extra
        fl[:] = self.flag
        return 0


def _truth(ds, qv, p, k):
    bp = pred.concat([p], N)
    ids, _, d32, cnt, _ = cpu.exact_topk(ds.vectors, ds.cols, qv[None], bp, k, threads=2)
    return ids[0][:cnt[0]], d32[0][:cnt[0]]


def _run_threads(fn, n):
    res = [None] * n
    ths = [threading.Thread(target=lambda i=i: res.__setitem__(i, fn(i))) for i in range(n)]
    for t in ths:
        t.start()
    for t in ths:
        t.join(30)
    return res


def test_concurrent_requests_batch_and_match_oracle(ds):
    preds = list(datagen.six_predicates().values())
    ex = OracleExec(ds)
    tids = (np.arange(N, dtype=np.uint64) * 7 + 1000)
    with Arbiter(nslots=64, batch_max=32, wait_us=3000, idle_us=2000) as a:
        a.set_executor(ex)
        a.attach(11, 77, count=N, dim=D, tids=tids)
        wants = [1, 5, 10, 17]

        def one(i):
            p = preds[i % len(preds)]
            return a.submit(11, 77, PV_STRAT_GPU_BRUTE, ds.queries[i], p, want=wants[i % 4])
        res = _run_threads(one, 48)
        st = a.stats()
    assert st["requests"] == 48 and st["batches"] < 48  # requests were gathered
    assert max(b["nq"] for b in ex.batches) > 1
    for i, (rc, hits, more) in enumerate(res):
        assert rc == 1
        ids, d = _truth(ds, ds.queries[i], preds[i % len(preds)], wants[i % 4])
        assert np.array_equal(hits["node"], ids.astype(np.uint64) * 7 + 1000)
        assert np.array_equal(hits["dist"], d)
        # the batch ran at its largest want: extra results set `more`
        if wants[i % 4] == 17:
            assert more == 0
    assert any(m for rc, h, m in res[::4])


def test_more_flags_and_prefix(ds):
    ex = OracleExec(ds, cnt_extra=3)  # the batch returned more than this slot asked
    with Arbiter(wait_us=0) as a:
        a.set_executor(ex)
        a.attach(1, 1, count=N, dim=D)
        rc, hits, more = a.submit(1, 1, PV_STRAT_GPU_BRUTE, ds.queries[0], None, want=4)
        assert rc == 1 and len(hits) == 4 and more == 1
        ex.cnt_extra, ex.flag = 0, 1  # truncated
        rc, hits, more = a.submit(1, 1, PV_STRAT_GPU_BRUTE, ds.queries[0], None, want=4)
        assert rc == 1 and more == 1
        ex.flag = 0
        rc, hits, more = a.submit(1, 1, PV_STRAT_GPU_BRUTE, ds.queries[0], None, want=4)
        assert rc == 1 and more == 0
        # graph: more unless exhausted
        rc, hits, more = a.submit(1, 1, PV_STRAT_GPU_HNSW, ds.queries[0], None, want=4)
        assert rc == 1 and more == 1
        ex.flag = 1
        rc, hits, more = a.submit(1, 1, PV_STRAT_GPU_HNSW, ds.queries[0], None, want=4)
        assert rc == 1 and more == 0


def test_out_of_range_rows_dropped(ds):
    ex = OracleExec(ds, bad_id_at=2)
    with Arbiter(wait_us=0) as a:
        a.set_executor(ex)
        a.attach(5, 9, count=N, dim=D)
        rc, hits, more = a.submit(5, 9, PV_STRAT_GPU_BRUTE, ds.queries[3], None, want=6)
    ids, _ = _truth(ds, ds.queries[3], None, 6)
    assert rc == 1 and len(hits) == 5
    assert np.array_equal(hits["node"], np.delete(ids, 2).astype(np.uint64))


def test_errors_and_capacity(ds):
    ex = OracleExec(ds)
    with Arbiter(wait_us=0) as a:
        a.set_executor(ex)
        a.attach(2, 3, count=N, dim=D)
        q = ds.queries[0]
        assert a.submit(2, 4, PV_STRAT_GPU_BRUTE, q, None, want=5)[0] == -1   # other file
        assert a.submit(2, 3, PV_STRAT_GPU_BRUTE, q[:8], None, want=5)[0] == -1  # dim
        assert a.submit(99, 3, PV_STRAT_GPU_BRUTE, q, None, want=5)[0] == -1  # not attached
        assert a.submit(2, 3, PV_STRAT_GPU_BRUTE, q, None, want=2000)[0] == 0  # capacity
        assert a.submit(2, 3, 7, q, None, want=5)[0] == 0  # not a GPU strategy
        big = pred.And(*[pred.Cmp(0, "<", float(i)) for i in range(60)])
        assert a.submit(2, 3, PV_STRAT_GPU_BRUTE, q, big, want=5)[0] == 0  # > 48 nodes
        ex.rc = -1
        assert a.submit(2, 3, PV_STRAT_GPU_BRUTE, q, None, want=5)[0] == -1  # batch failed
        assert len(ex.batches) == 1  # only the failing batch reached the executor


def test_graph_groups_heaviest_first_with_descended_entries(ds):
    h = Hnsw(ds.vectors, 8, 64, threads=2)
    ex = OracleExec(ds)
    gate = threading.Event()
    ex.gate = gate
    sels = [1000, 5, 200, 40, 1, 600]
    with Arbiter(wait_us=0) as a:
        a.set_executor(ex)
        a.attach(3, 1, count=N, dim=D, hnsw=h)
        # the first request holds the worker so that the other six queue
        # and form one batch
        t0 = threading.Thread(target=lambda: a.submit(3, 1, PV_STRAT_GPU_HNSW, ds.queries[40],
                                                      None, want=10, sel_permille=1000))
        t0.start()
        time.sleep(0.2)
        out = [None] * 6
        ths = [threading.Thread(target=lambda i=i: out.__setitem__(
            i, a.submit(3, 1, PV_STRAT_GPU_HNSW, ds.queries[i], None, want=10 + i,
                        max_visited=1000 * (i + 1), sel_permille=sels[i])))
            for i in range(6)]
        for t in ths:
            t.start()
        time.sleep(0.3)
        gate.set()
        for t in ths + [t0]:
            t.join(10)
    assert all(r[0] == 1 for r in out)
    b = ex.batches[1]
    assert b["nq"] == 6 and b["want"] == 15 and b["mv"] == 6000
    w = [(10 + i) * 1000.0 / max(sels[i], 1) for i in range(6)]
    order = sorted(range(6), key=lambda i: -w[i])
    # rows of the batch follow LPT order; each carries its descended entry
    for row, i in enumerate(order):
        assert np.array_equal(b["q"][row], ds.queries[i])
    assert np.array_equal(b["entries"], h.entries(ds.queries[order]))


def test_feedback_ewma(ds):
    ex = OracleExec(ds, delay=0.002)
    with Arbiter(wait_us=0) as a:
        a.set_executor(ex)
        a.attach(4, 1, count=N, dim=D)
        assert a.feedback(4, PV_STRAT_GPU_BRUTE) is None
        for sel in (500, 30, 1):
            assert a.submit(4, 1, PV_STRAT_GPU_BRUTE, ds.queries[0], None, want=3,
                            sel_permille=sel)[0] == 1
        f = a.feedback(4, PV_STRAT_GPU_BRUTE)
    assert f is not None
    assert f["q_us"][0] >= 2000 and f["q_us"][2] >= 2000 and f["q_us"][4] >= 2000
    assert f["q_us"][1] == 0 and f["q_us"][3] == 0
    assert f["batch_n16"] == 16 and f["batch_us"] >= 2000


def test_dead_worker_requests_reclaimed(ds):
    ex = OracleExec(ds)
    gate = threading.Event()
    ex.gate = gate
    with Arbiter(wait_us=0) as a:
        a.set_executor(ex)
        a.attach(6, 1, count=N, dim=D)
        res = [None] * 3
        ths = [threading.Thread(target=lambda i=i: res.__setitem__(
            i, a.submit(6, 1, PV_STRAT_GPU_BRUTE, ds.queries[i], None, want=5,
                        timeout_ms=5000))) for i in range(3)]
        for t in ths:
            t.start()
        time.sleep(0.2)
        a.kill_worker()  # the worker dies holding its batch
        gate.set()
        t = time.time()
        for th in ths:
            th.join(10)
        assert time.time() - t < 3
        assert all(r[0] == 0 for r in res)  # the callers keep their queries
        assert a.stats()["worker"] == 0 and a.stats()["inflight"] == 0
        # no worker: submit refuses at once
        assert a.submit(6, 1, PV_STRAT_GPU_BRUTE, ds.queries[0], None, want=5)[0] == 0


def test_stuck_worker_times_out_and_slot_is_reused(ds):
    ex = OracleExec(ds)
    gate = threading.Event()
    ex.gate = gate
    with Arbiter(nslots=2, wait_us=0) as a:
        a.set_executor(ex)
        a.attach(8, 1, count=N, dim=D)
        first = []
        t0 = threading.Thread(target=lambda: first.append(
            a.submit(8, 1, PV_STRAT_GPU_BRUTE, ds.queries[0], None, want=5)))
        t0.start()
        time.sleep(0.2)
        # the worker is busy: this request is never collected within 100 ms
        t = time.time()
        rc, _, _ = a.submit(8, 1, PV_STRAT_GPU_BRUTE, ds.queries[1], None, want=5,
                            timeout_ms=100)
        assert rc == 0 and time.time() - t < 2
        gate.set()
        t0.join(10)
        assert first[0][0] == 1
        # both slots are free again
        assert a.submit(8, 1, PV_STRAT_GPU_BRUTE, ds.queries[1], None, want=5)[0] == 1


def test_attach_while_serving_keeps_served_index_valid(ds):
    """pv_arbiter_attach may run beside the worker: a batch in flight keeps
    using its index's registration (tids, count) while hundreds of other
    indexes are attached, which used to reallocate the registry under it."""
    ex = OracleExec(ds)
    ex.gate = threading.Event()
    tids = np.arange(N, dtype=np.uint64) * 3 + 5
    q = ds.queries[0]
    with Arbiter(nslots=16, batch_max=8, wait_us=200, idle_us=100) as a:
        a.set_executor(ex)
        a.attach(1, 9, count=N, dim=D, tids=tids)
        out = {}
        t = threading.Thread(target=lambda: out.setdefault(
            "r", a.submit(1, 9, PV_STRAT_GPU_BRUTE, q, None, want=10)))
        t.start()
        time.sleep(0.05)  # the worker holds the batch at the gate
        for relid in range(100, 400):
            a.attach(relid, relid, count=N, dim=D, tids=tids)
        ex.gate.set()
        t.join(30)
        rc, hits, more = out["r"]
        ids, _ = _truth(ds, q, None, 10)
        assert rc == 1
        assert np.array_equal(hits["node"], ids.astype(np.uint64) * 3 + 5)
