"""The worker micro-batch loop driving the real GPU batch calls: requests
from many threads, gathered into batches, answered exactly as one direct
fv_gpu_brute_batch / fv_gpu_graph_batch call per request answers them."""
import threading

import numpy as np
import pytest

from paves_b200 import GpuIndex, datagen
from paves_b200.arbiter import PV_STRAT_GPU_BRUTE, PV_STRAT_GPU_HNSW, Arbiter
from paves_b200.hnsw import Hnsw

pytestmark = pytest.mark.gpu


def _threads(fn, n):
    res = [None] * n
    ths = [threading.Thread(target=lambda i=i: res.__setitem__(i, fn(i))) for i in range(n)]
    for t in ths:
        t.start()
    for t in ths:
        t.join(60)
    return res


def test_arbiter_brute_matches_direct_calls():
    n, d, nq = 40000, 64, 64
    ds = datagen.make_dataset(n, d, nq=nq)
    preds = list(datagen.six_predicates().values())
    g = GpuIndex(ds.vectors, ds.cols)
    tids = np.arange(n, dtype=np.uint64)[::-1].copy()
    wants = [1, 10, 32, 100]
    with Arbiter(nslots=128, batch_max=64, wait_us=2000, idle_us=500) as a:
        a.attach(7, 1, g, tids=tids)
        res = _threads(lambda i: a.submit(7, 1, PV_STRAT_GPU_BRUTE, ds.queries[i],
                                          preds[i % 6], want=wants[i % 4]), nq)
        st = a.stats()
    assert st["batches"] < nq
    for i, (rc, hits, more) in enumerate(res):
        assert rc == 1
        ids, dist, cnt, trunc = g.brute_batch(ds.queries[i:i + 1], [preds[i % 6]], wants[i % 4])
        c = int(cnt[0])
        assert np.array_equal(hits["node"], tids[ids[0][:c].astype(np.int64)])
        assert np.array_equal(hits["dist"], dist[0][:c])
    g.close()


def test_arbiter_graph_matches_direct_calls():
    n, d, nq = 20000, 32, 32
    ds = datagen.make_dataset(n, d, nq=nq)
    h = Hnsw(ds.vectors, 12, 100)
    g = GpuIndex(ds.vectors, ds.cols, l0=h.l0)
    p = datagen.graph_predicates()["sel10%"]
    with Arbiter(nslots=64, batch_max=64, wait_us=2000, idle_us=500) as a:
        a.attach(9, 1, g, hnsw=h)
        res = _threads(lambda i: a.submit(9, 1, PV_STRAT_GPU_HNSW, ds.queries[i], p, want=64,
                                          max_visited=200000, sel_permille=100), nq)
    ent = h.entries(ds.queries)
    ids, dist, cnt, exh = g.graph_batch(ds.queries, ent, [p] * nq, 64, 200000)
    for i, (rc, hits, more) in enumerate(res):
        assert rc == 1
        c = int(cnt[i])
        # the beam search of one query does not depend on its batch mates
        assert np.array_equal(hits["node"], ids[i][:c])
        assert np.array_equal(hits["dist"], dist[i][:c])
        assert more == (1 if exh[i] == 0 else 0)
    g.close()
