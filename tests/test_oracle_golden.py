"""Pins the oracle (oracle/paves_oracle.c) to the reference engine's own
outputs stored in tests/golden/ (generated by tests/golden/make_golden.py
from the reference sources). CPU only."""
import numpy as np

from oracle import cpu
from paves_b200 import pred


def test_exact_topk_matches_reference_brute_cursor(brute_golden):
    g = brute_golden
    nq = g["queries"].shape[0]
    for pi, p in enumerate(g["preds"]):
        bp = pred.concat([p] * nq, g["vectors"].shape[0])
        for k, ids_key, d_key in ((10, "ids10", "d10"), (100, "ids100", "d100")):
            ids, d64, d32, cnt, passing = cpu.exact_topk(g["vectors"], g["cols"], g["queries"],
                                                         bp, k)
            gid, gd = g[ids_key][pi], g[d_key][pi]
            for q in range(nq):
                n = int((gid[q] >= 0).sum())
                assert cnt[q] == n, (pi, k, q)
                assert np.array_equal(ids[q, :n].astype(np.int64), gid[q, :n]), (pi, k, q)
                # FP32 distances are exact on integer-valued rows
                assert np.array_equal(d32[q, :n], gd[q, :n]), (pi, k, q)
                assert np.array_equal(d64[q, :n].astype(np.float32), gd[q, :n])


def test_bitmap_matches_row_eval(brute_golden):
    g = brute_golden
    n = g["vectors"].shape[0]
    for p in g["preds"]:
        bp = pred.concat([p], n)
        words, npass = cpu.pred_bitmap(g["cols"], bp, 0)
        mask = pred.eval_numpy(p, g["cols"])
        bits = np.unpackbits(words.view(np.uint8), bitorder="little")[:n].astype(bool)
        assert np.array_equal(bits, mask)
        assert npass == mask.sum()


def test_hnsw_phase_matches_reference_cursor(graph_golden):
    g = graph_golden
    nq = g["queries"].shape[0]
    n = g["vectors"].shape[0]
    for pi, p in enumerate(g["preds"]):
        bp = pred.concat([p] * nq, n)
        for ei, ef in enumerate(g["efs"]):
            for q in range(nq):
                ids, dd, _ = cpu.hnsw_search(g["vectors"], g["l0"], int(g["entries"][q]),
                                             g["queries"][q], bp if p is not None else None, q,
                                             g["cols"], int(ef))
                gid = g["ids"][pi, ei, q]
                m = int((gid >= 0).sum())
                assert np.array_equal(ids[:m].astype(np.int64), gid[:m]), (pi, ef, q)
                assert np.array_equal(dd[:m], g["dists"][pi, ei, q, :m])


def test_graph_entry_matches_reference(graph_golden):
    from types import SimpleNamespace
    g = graph_golden
    f = SimpleNamespace(vectors=g["vectors"], dim=g["vectors"].shape[1],
                        upper_offs=g["upper_offs"], upper=g["upper"], M=int(g["M"]),
                        max_level=int(g["max_level"]), entry_node=int(g["entry_node"]))
    for q in range(g["queries"].shape[0]):
        assert cpu.graph_entry(f, g["queries"][q]) == int(g["entries"][q])
