"""Filtered level-0 beam search (fv_gpu_graph_batch through the C ABI)
against the reference HnswCursor's golden results and the exact scan.

Bar: every returned node passes its predicate, results are ascending by
(dist, node) with exact FP32 distances, and recall@10 against the exact
filtered top-10 is >= the reference beam search's recall at equal ef."""
import numpy as np
import pytest

from oracle import cpu
from paves_b200 import GpuError, GpuIndex, pred

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gidx(graph_golden):
    g = graph_golden
    return GpuIndex(g["vectors"], g["cols"], l0=g["l0"])


def recall(found, truth):
    t = set(int(x) for x in truth if x >= 0)
    if not t:
        return 1.0
    return len(t & set(int(x) for x in found[:10])) / len(t)


def test_recall_at_least_reference(gidx, graph_golden):
    g = graph_golden
    nq = g["queries"].shape[0]
    n = g["vectors"].shape[0]
    for pi, p in enumerate(g["preds"]):
        bp = pred.concat([p] * nq, n)
        truth = cpu.exact_topk(g["vectors"], g["cols"], g["queries"], bp, 10)[0]
        tcnt = cpu.exact_topk(g["vectors"], g["cols"], g["queries"], bp, 10)[3]
        mask = pred.eval_numpy(p, g["cols"])
        for ei, ef in enumerate(g["efs"]):
            ids, dists, cnt, exh = gidx.graph_batch(g["queries"], g["entries"], [p] * nq,
                                                    int(ef))
            r_gpu, r_ref = [], []
            for q in range(nq):
                c = int(cnt[q])
                got = ids[q, :c].astype(np.int64)
                assert mask[got].all(), "non-passing node returned"
                keys = list(zip(dists[q, :c].tolist(), got.tolist()))
                assert keys == sorted(keys)
                exact = np.sum((g["vectors"][got] - g["queries"][q]) ** 2, 1, dtype=np.float32)
                assert np.array_equal(exact, dists[q, :c])
                tr = truth[q, :tcnt[q]].astype(np.int64)
                r_gpu.append(recall(got, tr))
                r_ref.append(recall(g["ids"][pi, ei, q], tr))
            assert np.mean(r_gpu) >= np.mean(r_ref) - 1e-9, (pi, ef, np.mean(r_gpu),
                                                             np.mean(r_ref))


def test_exhausted_and_max_visited(gidx, graph_golden):
    g = graph_golden
    q = g["queries"][:4]
    e = g["entries"][:4]
    # tiny budget: stops early, flagged exhausted
    ids, dists, cnt, exh = gidx.graph_batch(q, e, [None] * 4, 16, max_visited=5)
    assert exh.tolist() == [1, 1, 1, 1]
    # impossible predicate: traversal runs until the frontier empties or
    # the budget is spent; no results, exhausted
    ids, dists, cnt, exh = gidx.graph_batch(q, e, [pred.Cmp(1, "<", -1.0)] * 4, 16)
    assert cnt.tolist() == [0, 0, 0, 0] and exh.tolist() == [1, 1, 1, 1]


def test_graph_errors(gidx, graph_golden):
    g = graph_golden
    q = g["queries"][:2]
    with pytest.raises(GpuError):
        gidx.graph_batch(q, [0, 0], [None, None], 0)
    with pytest.raises(GpuError):
        gidx.graph_batch(q, [0, 0], [None, None], 513)
    with pytest.raises(GpuError):
        gidx.graph_batch(q, [0, 10 ** 7], [None, None], 16)
    nog = GpuIndex(g["vectors"], g["cols"])
    with pytest.raises(GpuError):
        nog.graph_batch(q, [0, 0], [None, None], 16)
    nog.close()
    ids, dists, cnt, exh = gidx.graph_batch(q, g["entries"][:2], [None, None], 16)
    assert cnt.tolist() == [16, 16]
