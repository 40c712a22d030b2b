"""Generates tests/golden/*.npz from the REFERENCE engine itself.

Run in a container where the reference sources are present (they are
compiled by `make -C oracle ref` into oracle/_ref/):

    python tests/golden/make_golden.py

Fixtures:
  brute_golden.npz  N=20000 x 128 synthetic rows (seeded generator), 32
                    queries, a set of predicate shapes incl. NULL (NaN)
                    attribute values; reference BruteCursor top-10 and
                    top-100 ids + distances per (query, predicate).
  graph_golden.npz  N=4000 x 128 rows, HNSW built by the reference builder
                    (M=16, efC=200, one thread: deterministic), its
                    level-0 / upper sections, reference graph entries and
                    HnswCursor top-10 at ef in {16, 64} per predicate.
"""
from __future__ import annotations

import hashlib
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refengine  # noqa: E402
from paves_b200 import datagen  # noqa: E402
from paves_b200.indexfile import read_index  # noqa: E402
from tests.golden_preds import brute_predicates, graph_predicates  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def data_hash(*arrs):
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def make_brute():
    ds = datagen.make_dataset(20000, 128, nq=32)
    cols = ds.cols.copy()
    cols[datagen.COL_PRICE, ::37] = np.nan     # NULL prices
    cols[datagen.COL_CATEGORY, 5::53] = np.nan  # NULL categories
    preds = brute_predicates()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "b.idx")
        refengine.build_index(path, ds.vectors, cols, M=4, efc=16, threads=1)
        R = refengine.RefIndex(path)
        nq, npred = ds.queries.shape[0], len(preds)
        ids10 = np.zeros((npred, nq, 10), np.int64) - 1
        d10 = np.zeros((npred, nq, 10), np.float32)
        ids100 = np.zeros((npred, nq, 100), np.int64) - 1
        d100 = np.zeros((npred, nq, 100), np.float32)
        for pi, p in enumerate(preds):
            ph = R.compile(p)
            for q in range(nq):
                i, d = R.brute(ds.queries[q], ph, 10)
                ids10[pi, q, :len(i)] = i
                d10[pi, q, :len(i)] = d
                i, d = R.brute(ds.queries[q], ph, 100)
                ids100[pi, q, :len(i)] = i
                d100[pi, q, :len(i)] = d
            R.free_pred(ph)
        R.close()
    np.savez_compressed(os.path.join(OUT, "brute_golden.npz"), queries=ds.queries,
                        data_sha=data_hash(ds.vectors, cols), nan_price_step=37,
                        nan_cat_start=5, nan_cat_step=53, ids10=ids10, d10=d10, ids100=ids100,
                        d100=d100)


def make_graph():
    ds = datagen.make_dataset(4000, 128, nq=24)
    preds = graph_predicates()
    efs = [16, 64]
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "g.idx")
        refengine.build_index(path, ds.vectors, ds.cols, M=16, efc=200, threads=1)
        f = read_index(path)
        R = refengine.RefIndex(path)
        nq = ds.queries.shape[0]
        entries = np.array([R.graph_entry(ds.queries[q]) for q in range(nq)], np.uint32)
        ids = np.zeros((len(preds), len(efs), nq, 10), np.int64) - 1
        dd = np.zeros((len(preds), len(efs), nq, 10), np.float32)
        for pi, p in enumerate(preds):
            ph = R.compile(p)
            for ei, ef in enumerate(efs):
                for q in range(nq):
                    i, d = R.hnsw(ds.queries[q], ph, 10, ef)
                    ids[pi, ei, q, :len(i)] = i
                    dd[pi, ei, q, :len(i)] = d
            R.free_pred(ph)
        np.savez_compressed(os.path.join(OUT, "graph_golden.npz"), queries=ds.queries,
                            data_sha=data_hash(ds.vectors, ds.cols), l0=np.array(f.l0),
                            levels=np.array(f.levels), upper_offs=np.array(f.upper_offs),
                            upper=np.array(f.upper), M=f.M, max_level=f.max_level,
                            entry_node=f.entry_node, entries=entries, efs=np.array(efs),
                            ids=ids, dists=dd)
        R.close()


if __name__ == "__main__":
    make_brute()
    make_graph()
    for n in ("brute_golden.npz", "graph_golden.npz"):
        print(n, os.path.getsize(os.path.join(OUT, n)))
