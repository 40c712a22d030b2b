"""Labels and training for the learned router (paves_b200.router).

The method labels its own training queries: every query runs the scan
(exact top-k; the index's reduced-precision scan is exact on integer data
and re-ranked in FP32 otherwise) and the graph search at each ef of
router.EFS, and its label is the cheapest action whose recall@k reaches
the target — graph at the smallest sufficient ef when that search is
faster than the scan of a whole batch, else the scan.

    python -m paves_b200.router_train --rows 1000000 --queries 200000 \
        --out paves_b200/router_1m128.npz

builds the 1M x 128 mixture data set, its HNSW graph (M=16,
efConstruction=200) and 1024 k-means centroids, labels the queries on the
GPU, trains the MLP with the GPU kernels and writes the weights, feature
standardization and centroids.
"""
from __future__ import annotations

import argparse
import json
import time
from typing import List, Optional, Tuple

import numpy as np

from . import _lib, datagen, pred
from .index import GpuIndex
from .router import EFS, Router, init_params, kmeans, label_actions, recall_at

KS = (1, 5, 10, 20, 50, 100)


def random_predicates(rng: np.random.Generator, n: int) -> List[Optional[pred.Pred]]:
    """Filters of the six kinds with randomized constants (selectivity from
    about 0.02% to 100%): price < x (x log-uniform), category IN a random
    set, their conjunction, a price range, and no filter."""
    P, Cc = datagen.COL_PRICE, datagen.COL_CATEGORY
    out: List[Optional[pred.Pred]] = []
    for _ in range(n):
        t = rng.integers(0, 6)
        if t == 0:
            out.append(pred.Cmp(P, "<", float(np.exp(rng.uniform(np.log(1.0), np.log(1000.0))))))
        elif t == 1:
            cats = rng.choice(10, int(rng.integers(1, 10)), replace=False)
            out.append(pred.In(Cc, [float(c) for c in sorted(cats)]))
        elif t == 2:
            x = float(np.exp(rng.uniform(np.log(2.0), np.log(1000.0))))
            cats = rng.choice(10, int(rng.integers(1, 6)), replace=False)
            out.append(pred.And(pred.Cmp(P, "<", x), pred.In(Cc, [float(c) for c in sorted(cats)])))
        elif t == 3:
            a = float(rng.uniform(0, 900))
            out.append(pred.And(pred.Cmp(P, ">=", a),
                                pred.Cmp(P, "<", a + float(np.exp(rng.uniform(0, np.log(1000.0 - a + 1)))))))
        elif t == 4:
            out.append(pred.Cmp(Cc, "==", float(rng.integers(0, 10))))
        else:
            out.append(None)
    return out


def graph_stats(index: GpuIndex, nq: int) -> np.ndarray:
    st = np.zeros(nq * 4, np.uint32)
    _lib.lib().pv_graph_stats(index.handle, _lib.ptr(st), nq)
    return st.reshape(nq, 4)


def calibrate(index: GpuIndex, entries_fn, queries, preds, k: int = 10, nb: int = 64
              ) -> Tuple[float, float]:
    """(scan_ms, step_ms): device time of one nb-query scan batch, and the
    graph search's time per step (one wave of nb CTAs, longest query)."""
    L = _lib.lib()
    q = queries[:nb]
    p = preds[:nb]
    index.brute_batch(q, p, k)
    scan = []
    for _ in range(3):
        index.brute_batch(q, p, k)
        scan.append(L.pv_last_kernel_ms(index.handle))
    ent = entries_fn(q)
    per = []
    for ef in EFS:
        index.graph_batch(q, ent, p, ef)
        ms = L.pv_last_kernel_ms(index.handle)
        steps = graph_stats(index, nb)[:, 0].max()
        per.append(ms / max(int(steps), 1))
    return float(np.median(scan)), float(np.median(per))


def label_queries(index: GpuIndex, entries_fn, router: Router, queries: np.ndarray,
                  preds, ks: np.ndarray, scan_ms: float, step_ms: float,
                  target: float = 1.0, chunk: int = 1024):
    """-> feats [n][12], labels [n], recall [n][4], steps [n][4]."""
    n = len(queries)
    feats = np.zeros((n, 12), np.float32)
    recall = np.zeros((n, len(EFS)))
    steps = np.zeros((n, len(EFS)), np.uint32)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        q = queries[s:e]
        p = preds[s:e]
        k = ks[s:e]
        kmax = int(k.max())
        bp = pred.concat(p, index.count)
        feats[s:e] = router.features(index, q, bp, k)
        tid, _, tcnt, _ = index.brute_batch_raw(q, bp, kmax)
        ent = entries_fn(q)
        for ei, ef in enumerate(EFS):
            gid, _, gcnt, _ = index.graph_batch(q, ent, p, max(ef, kmax))
            steps[s:e, ei] = graph_stats(index, e - s)[:, 0]
            for kv in np.unique(k):
                sel = np.nonzero(k == kv)[0]
                recall[s + sel, ei] = recall_at(gid[sel], gcnt[sel], tid[sel],
                                                np.minimum(tcnt[sel], kv), int(kv))
    labels = label_actions(recall, steps * step_ms, scan_ms, target)
    return feats, labels, recall, steps


def standardization(feats: np.ndarray):
    mean = feats.mean(0).astype(np.float32)
    std = feats.std(0).astype(np.float32)
    std[std < 1e-6] = 1.0
    return mean, std


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=1_000_000)
    ap.add_argument("--dim", type=int, default=128)
    ap.add_argument("--queries", type=int, default=200_000)
    ap.add_argument("--centroids", type=int, default=1024)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--target", type=float, default=1.0)
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    from .hnsw import Hnsw
    t0 = time.time()
    ds = datagen.make_dataset(a.rows, a.dim, nq=16)
    h = Hnsw(ds.vectors, 16, 200)
    cent = kmeans(ds.vectors, a.centroids)
    index = GpuIndex(ds.vectors, ds.cols, l0=h.l0, precision=_lib.FV_GPU_PREC_BF16)
    router = Router(cent)
    rng = np.random.default_rng(datagen.SEED + 5)
    q = datagen.make_queries(ds.centers, a.queries, stream=5)
    preds = random_predicates(rng, a.queries)
    ks = rng.choice(np.asarray(KS, np.uint32), a.queries)
    print(json.dumps({"prep_s": round(time.time() - t0, 1)}), flush=True)
    scan_ms, step_ms = calibrate(index, h.entries, q, preds)
    feats, labels, recall, steps = label_queries(index, h.entries, router, q, preds, ks,
                                                 scan_ms, step_ms, a.target)
    print(json.dumps({"label_s": round(time.time() - t0, 1), "scan_ms": scan_ms,
                      "step_ms": step_ms,
                      "label_hist": np.bincount(labels, minlength=5).tolist()}), flush=True)
    mean, std = standardization(feats)
    router.set_params(init_params(1), mean, std)
    hist = router.train(feats, labels, epochs=a.epochs, batch=1024, lr=3e-3)
    acc = float((router.logits(feats).argmax(1) == labels).mean())
    print(json.dumps({"train_s": round(time.time() - t0, 1), "loss": hist.tolist()[-3:],
                      "train_acc": round(acc, 4)}), flush=True)
    np.savez(a.out, params=router.params(), mean=mean, std=std,
             centroids=cent.astype(np.float16), scan_ms=scan_ms, step_ms=step_ms,
             rows=a.rows, dim=a.dim, target=a.target)


if __name__ == "__main__":
    main()
