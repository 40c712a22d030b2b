"""Host HNSW builder (pv_hnsw_build) against the reference builder's output
in tests/golden/graph_golden.npz. CPU only."""
import os
import tempfile

import numpy as np

from oracle import cpu, refengine
from paves_b200 import datagen, pred
from paves_b200.hnsw import Hnsw
from paves_b200.indexfile import read_index


def test_single_thread_build_reproduces_reference_graph(graph_golden):
    g = graph_golden
    h = Hnsw(g["vectors"], 16, 200, threads=1)
    assert np.array_equal(h.levels, g["levels"])
    assert np.array_equal(h.l0, g["l0"])
    assert np.array_equal(h.upper_offs, g["upper_offs"])
    assert np.array_equal(h.upper, g["upper"])
    assert h.entry_node == int(g["entry_node"]) and h.max_level == int(g["max_level"])


def test_entries_match_reference_descent(graph_golden):
    g = graph_golden
    h = Hnsw(g["vectors"], 16, 200, threads=1)
    assert np.array_equal(h.entries(g["queries"], threads=3), g["entries"])


def test_parallel_build_quality():
    ds = datagen.make_dataset(6000, 64, nq=32)
    h = Hnsw(ds.vectors, 12, 100, threads=4)
    assert h.l0[:, 0].max() <= 24 and h.l0[:, 0].min() >= 1
    bp = pred.concat([None] * 32, 6000)
    truth = cpu.exact_topk(ds.vectors, ds.cols, ds.queries, bp, 10)[0]
    ent = h.entries(ds.queries)
    hit = 0
    for q in range(32):
        ids, _, _ = cpu.hnsw_search(ds.vectors, h.l0, int(ent[q]), ds.queries[q], None, q,
                                    ds.cols, 64)
        hit += len(set(ids[:10].tolist()) & set(truth[q].tolist()))
    assert hit / 320 >= 0.9


def test_written_file_serves_reference_cursor():
    ds = datagen.make_dataset(3000, 32, nq=8)
    h = Hnsw(ds.vectors, 8, 64, threads=2)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "h.idx")
        h.write(path, ds.cols)
        f = read_index(path)
        assert np.array_equal(f.l0, h.l0) and f.entry_node == h.entry_node
        if refengine.available("cpu"):
            R = refengine.RefIndex(path)
            p = datagen.graph_predicates()["sel10%"]
            ph = R.compile(p)
            bp = pred.concat([p] * 8, 3000)
            for q in range(8):
                rid, _ = R.hnsw(ds.queries[q], ph, 10, 32)
                assert R.graph_entry(ds.queries[q]) == int(h.entries(ds.queries[q:q + 1])[0])
                oid, _, _ = cpu.hnsw_search(ds.vectors, h.l0, R.graph_entry(ds.queries[q]),
                                            ds.queries[q], bp, q, ds.cols, 32)
                assert np.array_equal(rid, oid[:10].astype(np.uint64))
            R.free_pred(ph)
            R.close()
