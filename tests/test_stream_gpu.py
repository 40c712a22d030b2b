"""Uneven micro-batches through the stream's CUDA graphs: per-query k and
filters, padding to the bucket, autotuned plans saved and reloaded,
predicate overflow through the ordinary path; results against the
oracle's exact filtered top-k."""
import os
import tempfile

import numpy as np
import pytest

from oracle import cpu
from paves_b200 import GpuIndex, _lib, datagen, pred
from paves_b200.stream import Stream

pytestmark = pytest.mark.gpu
N, D = 60000, 96


def random_filter(rng):
    P, Cc = datagen.COL_PRICE, datagen.COL_CATEGORY
    sel = np.exp(rng.uniform(np.log(0.0005), np.log(0.9)))
    a = float(rng.uniform(0, 1000 * (1 - min(sel, 0.9))))
    p = pred.And(pred.Cmp(P, ">=", a), pred.Cmp(P, "<", a + 1000 * sel))
    if rng.random() < 0.3:
        p = pred.And(p, pred.In(Cc, [float(c) for c in sorted(rng.choice(10, 5, replace=False))]))
    return p


@pytest.fixture(scope="module")
def env():
    ds = datagen.make_dataset(N, D, nq=256, ncomp=256)
    g = GpuIndex(ds.vectors, ds.cols, precision=_lib.FV_GPU_PREC_FP8)
    td = tempfile.mkdtemp()
    path = os.path.join(td, "tune.txt")
    s = Stream(g, 64, 100, ds.queries[:64], path)
    yield ds, g, s, path
    s.close()
    g.close()


def _check(ds, q, preds, k, ids, dists, cnt):
    bp = pred.concat(preds, N)
    o_ids, _, _, o_cnt, _ = cpu.exact_topk(ds.vectors, ds.cols, q, bp, int(np.max(k)))
    hit = tot = 0
    for i in range(len(q)):
        kk = int(k[i])
        t = o_ids[i, :min(kk, int(o_cnt[i]))]
        assert cnt[i] == len(t)
        hit += np.isin(t, ids[i, :cnt[i]]).sum()
        tot += len(t)
        rows = ids[i, :cnt[i]].astype(np.int64)
        exact = np.sum((ds.vectors[rows] - q[i]) ** 2, 1, dtype=np.float32)
        assert np.array_equal(dists[i, :cnt[i]], exact)
        assert np.all(np.diff(dists[i, :cnt[i]]) >= 0)
    return hit / max(tot, 1)


def test_uneven_batches_mixed_k_and_filters(env):
    ds, g, s, path = env
    rng = np.random.default_rng(4)
    plans = s.plans()
    assert {p["batch"] for p in plans} == {1, 2, 4, 8, 16, 32, 64}
    hits = []
    for nq in (1, 3, 17, 64, 5):
        idx = rng.choice(256, nq, replace=False)
        q = ds.queries[idx]
        preds = [random_filter(rng) for _ in range(nq)]
        k = rng.choice(np.array([1, 10, 100], np.uint32), nq)
        ids, dists, cnt, ms = s.run(q, preds, k)
        assert ms > 0 and s.last()["fallback"] == 0
        hits.append(_check(ds, q, preds, k, ids, dists, cnt))
    assert np.mean(hits) >= 0.98, hits


def test_tuning_file_reloads(env):
    ds, g, s, path = env
    assert os.path.exists(path)
    s2 = Stream(g, 64, 100, ds.queries[:64], path)
    assert [ {k: v for k, v in p.items() if k != "tuned_ms"} for p in s2.plans()] == \
        [{k: v for k, v in p.items() if k != "tuned_ms"} for p in s.plans()]
    q = ds.queries[:7]
    preds = [None] * 7
    a = s.run(q, preds, 10)
    b = s2.run(q, preds, 10)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
    s2.close()


def test_predicate_overflow_takes_the_ordinary_path(env):
    ds, g, s, path = env
    # 100 distinct values, not all small integers: stays a 100-constant IN list
    big = pred.In(datagen.COL_CATEGORY, [float(c) for c in range(10)] +
                  [100.5 + c for c in range(90)])
    q = ds.queries[:1]
    ids, dists, cnt, ms = s.run(q, [big], 10)
    assert s.last()["fallback"] == 1
    assert _check(ds, q, [big], np.array([10]), ids, dists, cnt) >= 0.99


def test_lazy_and_bitmap_filters_in_one_stream(env):
    """Batches whose filters are all ranges / small-integer sets are tested
    lazily inside the scan (no bitmaps); a batch with an OR or NOT filter
    takes the bitmaps. Both must give the oracle's answers, also when they
    alternate on the same captured graph."""
    ds, g, s, path = env
    rng = np.random.default_rng(11)
    P, Cc = datagen.COL_PRICE, datagen.COL_CATEGORY
    orf = pred.Or(pred.Cmp(P, "<", 30.0), pred.In(Cc, [2.0]))
    notf = pred.Not(pred.Cmp(P, "<", 900.0))
    for rep in range(3):
        for mix in ("lazy", "bitmap"):
            nq = 16
            q = ds.queries[rng.choice(256, nq, replace=False)]
            preds = [random_filter(rng) for _ in range(nq)]
            if mix == "bitmap":
                preds[3] = orf
                preds[9] = notf
            k = rng.choice(np.array([1, 10, 100], np.uint32), nq)
            ids, dists, cnt, ms = s.run(q, preds, k)
            assert s.last()["fallback"] == 0
            assert _check(ds, q, preds, k, ids, dists, cnt) >= 0.98, (rep, mix)
