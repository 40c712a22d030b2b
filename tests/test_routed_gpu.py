"""pv_routed_batch: the router's decisions drive one scan or one graph
search per batch, with results identical to the direct entry points."""
import numpy as np
import pytest

from paves_b200 import GpuIndex, _lib, datagen
from paves_b200.hnsw import Hnsw
from paves_b200.router import Router, init_params, kmeans, routed_batch

pytestmark = pytest.mark.gpu
N, D, NQ = 60000, 64, 64


@pytest.fixture(scope="module")
def env():
    ds = datagen.make_dataset(N, D, nq=NQ)
    h = Hnsw(ds.vectors, 12, 100)
    g = GpuIndex(ds.vectors, ds.cols, l0=h.l0, precision=_lib.FV_GPU_PREC_BF16)
    cent = kmeans(ds.vectors, 64, iters=4, sample=8192)
    r = Router(cent)
    yield ds, h, g, r
    r.close()
    g.close()


def _preds():
    six = list(datagen.six_predicates().values())
    return [six[i % 6] for i in range(NQ)]


def test_plan_scan_equals_brute(env):
    ds, h, g, r = env
    preds = _preds()
    ent = h.entries(ds.queries)
    k = np.array([[1, 10, 32][i % 3] for i in range(NQ)], np.uint32)
    ids, dist, cnt, dec, ex, st = routed_batch(g, None, ds.queries, preds, k, ent, topb=32,
                                               plan=np.zeros(NQ, np.uint16))
    assert ex == 0 and (dec == 0).all()
    bi, bd, bc, _ = g.brute_batch(ds.queries, preds, 32)
    for i in range(NQ):
        c = min(int(bc[i]), int(k[i]))
        assert cnt[i] == c
        assert np.array_equal(ids[i, :c], bi[i, :c]) and np.array_equal(dist[i, :c], bd[i, :c])


def test_plan_graph_equals_graph_batch(env):
    ds, h, g, r = env
    preds = _preds()
    ent = h.entries(ds.queries)
    k = np.full(NQ, 10, np.uint32)
    plan = np.array([[32, 64, 128][i % 3] for i in range(NQ)], np.uint16)
    ids, dist, cnt, dec, ex, st = routed_batch(g, None, ds.queries, preds, k, ent, plan=plan)
    assert ex == 1 and np.array_equal(dec, plan)
    for ef in (32, 64, 128):
        sel = np.nonzero(plan == ef)[0]
        gi, gd, gc, _ = g.graph_batch(ds.queries[sel], ent[sel], [preds[i] for i in sel], ef)
        for j, i in enumerate(sel):
            c = min(int(gc[j]), 10)
            assert cnt[i] == c
            assert np.array_equal(ids[i, :c], gi[j, :c])
            assert np.array_equal(dist[i, :c], gd[j, :c])


def test_mixed_plan_scans_and_router_decisions(env):
    ds, h, g, r = env
    preds = _preds()
    ent = h.entries(ds.queries)
    k = np.full(NQ, 10, np.uint32)
    plan = np.full(NQ, 64, np.uint16)
    plan[5] = 0
    plan[11] = 0
    ids, dist, cnt, dec, ex, st = routed_batch(g, None, ds.queries, preds, k, ent, plan=plan)
    assert ex == 0  # a scanned batch answers every query from the scan
    bi, bd, bc, _ = g.brute_batch(ds.queries, preds, 10)
    assert np.array_equal(ids, bi) and np.array_equal(dist, bd)
    ids, dist, cnt, dec, ex, st = routed_batch(g, None, ds.queries, preds, k, ent, plan=plan,
                                               split=True)
    assert ex == 2  # split: each query takes its own route
    bi, bd, bc, _ = g.brute_batch(ds.queries, preds, 10)
    sc = plan == 0
    assert np.array_equal(ids[sc], bi[sc]) and np.array_equal(dist[sc], bd[sc])
    gsel = np.nonzero(plan > 0)[0]
    gi, gd, gc, _ = g.graph_batch(ds.queries[gsel], ent[gsel], [preds[i] for i in gsel], 64)
    for j, i in enumerate(gsel):
        c = min(int(gc[j]), 10)
        assert cnt[i] == c
        assert np.array_equal(ids[i, :c], gi[j, :c]) and np.array_equal(dist[i, :c], gd[j, :c])
    # learned decisions equal the host rule applied to the router's logits
    rng = np.random.default_rng(2)
    p = init_params(4)
    p[-5:] = rng.standard_normal(5).astype(np.float32)
    from paves_b200 import pred
    f = r.features(g, ds.queries, pred.concat(preds, N), k)
    r.set_params(p, f.mean(0), f.std(0) + 1e-3)
    for margin in (0.0, 0.3):
        ids, dist, cnt, dec, ex, st = routed_batch(g, r, ds.queries, preds, k, ent,
                                                   margin=margin)
        a = r.decide(f, k, margin)
        want = np.where(a == 0, 0, np.maximum(np.array([0, 32, 64, 128, 256])[a], 10))
        assert np.array_equal(dec, want.astype(np.uint16))
        assert ex == (1 if (want > 0).all() else 0)
        assert (st >= 0).all()
