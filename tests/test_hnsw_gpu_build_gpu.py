"""The GPU HNSW builder (pv_hnsw_build_gpu): a valid graph in the index
file's layout, and filtered search recall on it at least the recall on the
host builder's graph (the engine's own construction, engine.cpp:698-1032)
at equal ef — the contract of a graph, since the two graphs differ.

Recall@10 is against the exact filtered top-10; the search is this
library's fv_gpu_graph_batch with the engine's default max_visited, and
also the reference engine's own HnswCursor on the file written from the
GPU-built sections (the file opens in the engine)."""
import os
import tempfile

import numpy as np
import pytest

from oracle import cpu, refengine
from paves_b200 import GpuIndex, datagen, pred
from paves_b200.hnsw import Hnsw

pytestmark = pytest.mark.gpu
N, D, NQ, M = 60_000, 128, 64, 16


@pytest.fixture(scope="module")
def graphs():
    ds = datagen.make_dataset(N, D, nq=NQ)
    hg = Hnsw(ds.vectors, M, builder="gpu")
    hh = Hnsw(ds.vectors, M, 200)
    return ds, hg, hh


def test_structure(graphs):
    ds, hg, hh = graphs
    l0 = hg.l0
    assert l0.shape == (N, 2 * M + 1)
    cnt = l0[:, 0]
    assert cnt.max() <= 2 * M and cnt.min() >= 1
    assert np.mean(cnt) > M  # lists mostly filled
    for i in range(0, N, 997):
        nb = l0[i, 1:1 + cnt[i]]
        assert np.all(nb < N) and i not in nb and len(set(nb.tolist())) == len(nb)
    assert np.array_equal(hg.levels, hh.levels)  # same level draw
    top = int(hg.levels.max())
    assert hg.max_level == top and hg.levels[hg.entry_node] == top
    assert hg.entry_node == int(np.flatnonzero(hg.levels == top)[0])
    # upper lists: neighbours are nodes of that level
    for i in np.flatnonzero(hg.levels >= 1)[:300]:
        for lv in range(1, int(hg.levels[i]) + 1):
            o = int(hg.upper_offs[i]) + (lv - 1) * (M + 1)
            c = int(hg.upper[o])
            nb = hg.upper[o + 1:o + 1 + c]
            assert c <= M and np.all(hg.levels[nb] >= lv) and i not in nb


def _recall(ids, cnt, truth, tcnt):
    r = []
    for i in range(len(cnt)):
        t = truth[i, :tcnt[i]]
        if len(t) == 0:
            continue
        r.append(np.isin(t, ids[i, :cnt[i]]).mean())
    return float(np.mean(r))


def test_recall_at_least_host_graph(graphs):
    ds, hg, hh = graphs
    q = ds.queries
    res = {}
    for name, h in (("gpu", hg), ("host", hh)):
        gi = GpuIndex(ds.vectors, ds.cols, l0=h.l0)
        ent = h.entries(q)
        for fname, p in datagen.graph_predicates().items():
            bp = pred.concat([p] * NQ, N)
            truth, _, _, tcnt, _ = cpu.exact_topk(ds.vectors, ds.cols, q, bp, 10)
            for ef in (32, 64, 128):
                ids, _, cnt, _ = gi.graph_batch(q, ent, [p] * NQ, ef)
                res[(name, fname, ef)] = _recall(ids, np.minimum(cnt, 10), truth, tcnt)
        gi.close()
    print({f"{k[0]}/{k[1]}/ef{k[2]}": round(v, 4) for k, v in res.items()})
    g = np.mean([v for k, v in res.items() if k[0] == "gpu"])
    hst = np.mean([v for k, v in res.items() if k[0] == "host"])
    assert g >= hst - 0.005, (g, hst)
    for fname in datagen.graph_predicates():
        for ef in (64, 128):
            assert res[("gpu", fname, ef)] >= res[("host", fname, ef)] - 0.02, (fname, ef, res)


def test_file_opens_in_the_engine(graphs):
    ds, hg, hh = graphs
    if not refengine.available("cpu"):
        pytest.skip("reference engine not built")
    td = tempfile.mkdtemp(dir="/tmp")
    path = os.path.join(td, "gpu_graph.idx")
    hg.write(path, ds.cols)
    R = refengine.RefIndex(path)
    p = datagen.graph_predicates()["sel10%"]
    ph = R.compile(p)
    bp = pred.concat([p] * 16, N)
    truth, _, _, tcnt, _ = cpu.exact_topk(ds.vectors, ds.cols, ds.queries[:16], bp, 10)
    rec = []
    for i in range(16):
        assert R.graph_entry(ds.queries[i]) == int(hg.entries(ds.queries[i:i + 1])[0])
        ids, _ = R.hnsw(ds.queries[i], ph, 10, 128)
        rec.append(np.isin(truth[i, :tcnt[i]], ids).mean())
    assert np.mean(rec) >= 0.9, rec
    R.free_pred(ph)
    R.close()
    os.unlink(path)
    os.rmdir(td)
