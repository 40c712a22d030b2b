"""The persistent micro-batch kernel (pv_serve_*): uneven batches with a k
and a filter per query against the oracle's exact filtered top-k, on the
lazy-filter and the bitmap phase; its bounded waits made to run out with
no fault: the queue wait (the kernel leaves after idle_ms and the next
batch starts it again) and a grid barrier whose arrival is withheld on
purpose (the batch call returns -1, and the next batch is served)."""
import time

import numpy as np
import pytest

from oracle import cpu
from paves_b200 import GpuIndex, _lib, datagen, pred
from paves_b200.stream import Serve

pytestmark = pytest.mark.gpu
N, D = 60000, 96


def random_filter(rng, broad=False):
    P, Cc = datagen.COL_PRICE, datagen.COL_CATEGORY
    lo_sel = np.log(0.3) if broad else np.log(0.0005)
    sel = np.exp(rng.uniform(lo_sel, np.log(0.9)))
    a = float(rng.uniform(0, 1000 * (1 - min(sel, 0.9))))
    p = pred.And(pred.Cmp(P, ">=", a), pred.Cmp(P, "<", a + 1000 * sel))
    if not broad and rng.random() < 0.3:
        p = pred.And(p, pred.In(Cc, [float(c) for c in sorted(rng.choice(10, 5, replace=False))]))
    return p


@pytest.fixture(scope="module")
def env():
    ds = datagen.make_dataset(N, D, nq=512, ncomp=256)
    g = GpuIndex(ds.vectors, ds.cols, precision=_lib.FV_GPU_PREC_FP8)
    s = Serve(g, 256, 100, idle_ms=500)
    yield ds, g, s
    s.close()
    g.close()


def _check(ds, q, preds, k, ids, dists, cnt, exact=False):
    bp = pred.concat(preds, N)
    o_ids, _, o_d32, o_cnt, _ = cpu.exact_topk(ds.vectors, ds.cols, q, bp, int(np.max(k)))
    hit = tot = 0
    for i in range(len(q)):
        kk = int(k[i])
        t = o_ids[i, :min(kk, int(o_cnt[i]))]
        assert cnt[i] == len(t), i
        hit += np.isin(t, ids[i, :cnt[i]]).sum()
        tot += len(t)
        rows = ids[i, :cnt[i]].astype(np.int64)
        assert np.array_equal(dists[i, :cnt[i]],
                              np.sum((ds.vectors[rows] - q[i]) ** 2, 1, dtype=np.float32))
        assert np.all(np.diff(dists[i, :cnt[i]]) >= 0)
        if exact:
            assert np.array_equal(ids[i, :cnt[i]], t.astype(np.uint64)), i
    return hit / max(tot, 1)


def test_uneven_batches_mixed_k_and_filters(env):
    ds, g, s = env
    rng = np.random.default_rng(4)
    hits = []
    for nq, broad in ((1, False), (3, True), (17, False), (64, True), (130, False), (5, False),
                      (256, True)):
        q = ds.queries[rng.choice(512, nq, replace=False)]
        preds = [random_filter(rng, broad) for _ in range(nq)]
        k = rng.choice(np.array([1, 10, 100], np.uint32), nq)
        ids, dists, cnt, ms = s.run(q, preds, k)
        st = s.status()
        assert ms > 0 and st["fallback"] == 0 and st["running"] == 1
        hits.append(_check(ds, q, preds, k, ids, dists, cnt))
    assert np.mean(hits) >= 0.98, hits
    assert s.status()["batches"] >= 7


def test_integer_rows_bf16_exact():
    ds = datagen.make_dataset(40_000, 128, nq=64)
    g = GpuIndex(ds.vectors, ds.cols, precision=_lib.FV_GPU_PREC_BF16)
    s = Serve(g, 64, 16, idle_ms=200)
    six = list(datagen.six_predicates().values()) + [None]
    preds = [six[i % len(six)] for i in range(64)]
    for rep in range(2):
        ids, dists, cnt, ms = s.run(ds.queries, preds, 10)
        _check(ds, ds.queries, preds, np.full(64, 10), ids, dists, cnt, exact=True)
    s.close()
    g.close()


def test_queue_wait_expires_and_restarts(env):
    ds, g, s = env
    rng = np.random.default_rng(9)
    s.limits(idle_ms=30, barrier_ms=2000)
    q = ds.queries[:8]
    preds = [random_filter(rng) for _ in range(8)]
    s.run(q, preds, 10)
    time.sleep(0.3)  # no batch: the kernel's wait for the next one runs out
    st = s.status()
    assert st["running"] == 0 and st["last_exit"] == 1, st
    ids, dists, cnt, ms = s.run(q, preds, 10)  # started again
    assert s.status()["running"] == 1
    _check(ds, q, preds, np.full(8, 10), ids, dists, cnt)
    s.limits(idle_ms=500, barrier_ms=2000)


def test_withheld_barrier_arrival_fails_the_batch_then_recovers(env):
    ds, g, s = env
    rng = np.random.default_rng(13)
    q = ds.queries[8:24]
    preds = [random_filter(rng) for _ in range(16)]
    s.limits(idle_ms=50, barrier_ms=50, skip_cta=3)
    with pytest.raises(RuntimeError, match="wait .*expired"):
        s.run(q, preds, 10)
    assert s.status()["last_exit"] == -1
    s.limits(idle_ms=500, barrier_ms=2000)
    ids, dists, cnt, ms = s.run(q, preds, 10)
    _check(ds, q, preds, np.full(16, 10), ids, dists, cnt)
