"""Learned scan-vs-graph router (libpaves_gpu.so ``pv_router_*``) and the
plain rule it stands beside.

Actions: 0 = scan (the index's brute path), 1..4 = graph beam search at
ef 32, 64, 128, 256 (``EFS``).

* ``kmeans``: the router's centroids (host, numpy; offline preparation).
* ``Router``: device-resident centroids + MLP; ``features`` runs the GPU
  features kernel, ``logits`` the bf16 MLP, ``grad`` / ``train`` the
  training kernels.
* ``plain_rule``: the reference's routing and beam width — the GPU path
  cost of planner.c:228-263 (gpu_path_cost_ms) priced from the worker's
  feedback EWMAs, and the selectivity-scaled ef of exec.c:415-424.
* ``make_labels``: labels the method generates for itself — for every
  query the exact top-k (scan) and the graph search at each ef, and the
  cheapest action that reaches the recall target.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import PV_MLP_IN, PV_MLP_NPARAMS, PV_MLP_OUT, ptr
from .pred import BatchPred

EFS = (32, 64, 128, 256)
NACT = PV_MLP_OUT


def _err():
    return C.create_string_buffer(512)


def kmeans(x: np.ndarray, k: int = 1024, iters: int = 8, sample: int = 131072,
           seed: int = 20240617 + 11) -> np.ndarray:
    """Lloyd's k-means on a seeded sample of the rows -> [k][d] float32."""
    rng = np.random.default_rng(seed)
    x = np.asarray(x, np.float32)
    s = x[rng.choice(len(x), min(sample, len(x)), replace=False)]
    c = s[rng.choice(len(s), k, replace=False)].copy()
    sn = (s * s).sum(1)
    for _ in range(iters):
        d = sn[:, None] - 2.0 * (s @ c.T) + (c * c).sum(1)[None, :]
        a = d.argmin(1)
        cnt = np.bincount(a, minlength=k).astype(np.float32)
        tot = np.zeros_like(c)
        np.add.at(tot, a, s)
        nz = cnt > 0
        c[nz] = tot[nz] / cnt[nz, None]
    return c


LAYOUT = (("W1", (12, 64)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)),
          ("W3", (64, 5)), ("b3", (5,)))  # order of the flat parameter vector


def init_params(seed: int = 1) -> np.ndarray:
    """He-initialized weights, zero biases (flat, LAYOUT order)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shp in LAYOUT:
        if name.startswith("W"):
            parts.append(rng.standard_normal(shp).ravel() * np.sqrt(2.0 / shp[0]))
        else:
            parts.append(np.zeros(shp[0]))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == PV_MLP_NPARAMS
    return p


class Router:
    def __init__(self, centroids: np.ndarray, device: int = 0):
        self._L = _lib.lib()
        self.centroids = np.ascontiguousarray(centroids, np.float32)
        err = _err()
        h = self._L.pv_router_create(device, ptr(self.centroids), self.centroids.shape[0],
                                     self.centroids.shape[1], err, len(err))
        if not h:
            raise RuntimeError(err.value.decode())
        self._h = h
        self.mean = np.zeros(PV_MLP_IN, np.float32)
        self.std = np.ones(PV_MLP_IN, np.float32)

    def close(self):
        if getattr(self, "_h", None):
            self._L.pv_router_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params: np.ndarray, mean: np.ndarray, std: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == PV_MLP_NPARAMS
        self.mean = np.ascontiguousarray(mean, np.float32)
        self.std = np.ascontiguousarray(std, np.float32)
        err = _err()
        if self._L.pv_router_set_params(self._h, ptr(p), ptr(self.mean), ptr(self.std), err,
                                        len(err)) != 0:
            raise RuntimeError(err.value.decode())

    def params(self) -> np.ndarray:
        p = np.zeros(PV_MLP_NPARAMS, np.float32)
        m = np.zeros(PV_MLP_IN, np.float32)
        s = np.zeros(PV_MLP_IN, np.float32)
        if self._L.pv_router_get_params(self._h, ptr(p), ptr(m), ptr(s)) != 0:
            raise RuntimeError("pv_router_get_params failed")
        return p

    def features(self, index, queries: np.ndarray, bp: BatchPred, k) -> np.ndarray:
        q = np.ascontiguousarray(queries, np.float32)
        nq = q.shape[0]
        kk = np.ascontiguousarray(np.broadcast_to(np.asarray(k, np.uint32), (nq,)))
        out = np.zeros((nq, PV_MLP_IN), np.float32)
        err = _err()
        rc = self._L.pv_router_features(self._h, index.handle, nq, ptr(q), ptr(bp.qd),
                                        ptr(bp.nodes), len(bp.nodes), ptr(bp.children),
                                        len(bp.children), ptr(bp.invals), len(bp.invals),
                                        ptr(kk), ptr(out), err, len(err))
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return out

    def logits(self, feats: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(feats, np.float32)
        out = np.zeros((f.shape[0], NACT), np.float32)
        err = _err()
        if self._L.pv_router_forward(self._h, f.shape[0], ptr(f), ptr(out), err, len(err)) != 0:
            raise RuntimeError(err.value.decode())
        return out

    def grad(self, feats, labels, sample_w=None):
        f = np.ascontiguousarray(feats, np.float32)
        y = np.ascontiguousarray(labels, np.int32)
        w = None if sample_w is None else np.ascontiguousarray(sample_w, np.float32)
        g = np.zeros(PV_MLP_NPARAMS, np.float32)
        loss = C.c_float()
        err = _err()
        if self._L.pv_router_grad(self._h, f.shape[0], ptr(f), ptr(y), ptr(w), ptr(g),
                                  C.byref(loss), err, len(err)) != 0:
            raise RuntimeError(err.value.decode())
        return float(loss.value), g

    def train(self, feats, labels, sample_w=None, epochs: int = 20, batch: int = 1024,
              lr: float = 3e-3, seed: int = 7) -> np.ndarray:
        f = np.ascontiguousarray(feats, np.float32)
        y = np.ascontiguousarray(labels, np.int32)
        w = None if sample_w is None else np.ascontiguousarray(sample_w, np.float32)
        hist = np.zeros(epochs, np.float32)
        err = _err()
        if self._L.pv_router_train(self._h, f.shape[0], ptr(f), ptr(y), ptr(w), epochs, batch,
                                   lr, seed, ptr(hist), err, len(err)) != 0:
            raise RuntimeError(err.value.decode())
        return hist

    def decide(self, feats: np.ndarray, k, margin: float = 0.0) -> np.ndarray:
        """Action per query: the most probable one, except that a graph
        action whose probability does not beat scan by `margin` yields to
        scan (margin > 0 trades speed for recall)."""
        z = self.logits(feats)
        p = np.exp(z - z.max(1, keepdims=True))
        p /= p.sum(1, keepdims=True)
        a = p.argmax(1)
        weak = (a > 0) & (p[np.arange(len(a)), a] < p[:, 0] + margin)
        a[weak] = 0
        return a


def ef_of(action: np.ndarray, k) -> np.ndarray:
    """Beam width of a graph action (never below k)."""
    efs = np.asarray((0,) + EFS)
    return np.maximum(efs[np.asarray(action)], np.asarray(k))


# ---------------------------------------------------------------- plain rule
FV_GPU_FIXED_MS = 0.4
FV_GPU_SEED_BRUTE_MS = 1.0
FV_GPU_SEED_GRAPH_MS = 0.5
SEL_MID = (0.40, 0.10, 0.022, 0.0045, 0.001)


def sel_bucket(permille: int) -> int:
    """arbiter.h:50-60 fv_sel_bucket."""
    if permille >= 200:
        return 0
    if permille >= 50:
        return 1
    if permille >= 10:
        return 2
    if permille >= 2:
        return 3
    return 4


@dataclass
class Feedback:
    """The worker's EWMAs for one index (arbiter.h:80-97), in us; 0 = none."""
    q_us: np.ndarray            # [2][5]: brute, graph per selectivity bucket
    batch_us: np.ndarray        # [2]
    batch_n16: np.ndarray       # [2]

    @staticmethod
    def empty() -> "Feedback":
        return Feedback(np.zeros((2, 5), np.uint32), np.zeros(2, np.uint32),
                        np.zeros(2, np.uint32))


def _nearest(row, b):
    for d in range(5):
        if b - d >= 0 and row[b - d]:
            return int(row[b - d]), b - d
        if b + d < 5 and row[b + d]:
            return int(row[b + d]), b + d
    return 0, b


def gpu_path_cost_ms(fb: Optional[Feedback], graph: bool, sel: float,
                     inflight: float = 0.0) -> float:
    """planner.c:228-263: fixed round trip + own amortized service time
    (observed per bucket, rescaled across buckets for the graph) + batch
    time x batches queued ahead."""
    si = 1 if graph else 0
    b = sel_bucket(int(sel * 1000))
    q_ms = FV_GPU_SEED_GRAPH_MS if graph else FV_GPU_SEED_BRUTE_MS
    navg = 1.0
    if fb is not None:
        q, src = _nearest(fb.q_us[si], b)
        if q:
            q_ms = q / 1000.0
            if si == 1 and src != b:
                q_ms *= SEL_MID[src] / SEL_MID[b]
        if fb.batch_n16[si]:
            navg = max(fb.batch_n16[si] / 16.0, 1.0)
        batch_ms = fb.batch_us[si] / 1000.0 if fb.batch_us[si] else q_ms
    else:
        batch_ms = q_ms
    return FV_GPU_FIXED_MS + q_ms + batch_ms * (inflight / navg)


def plain_rule(sel: np.ndarray, k: np.ndarray, fb: Optional[Feedback] = None,
               ef_search: int = 100):
    """-> (graph? bool[nq], ef int[nq]): the cheaper GPU strategy by the
    planner's cost, and exec.c's ef = max(k, ef_search x {1, 0.8, 0.4} by
    selectivity >= 0.4 / >= 0.15 / else)."""
    sel = np.asarray(sel, np.float64)
    k = np.asarray(k)
    graph = np.array([gpu_path_cost_ms(fb, True, s) < gpu_path_cost_ms(fb, False, s)
                      for s in sel], bool)
    scale = np.where(sel >= 0.4, 1.0, np.where(sel >= 0.15, 0.8, 0.4))
    ef = np.maximum(k, (ef_search * scale).astype(np.int64))
    return graph, ef


# ---------------------------------------------------------------- labels
def recall_at(found_ids: np.ndarray, found_cnt, truth_ids: np.ndarray, truth_cnt, k: int):
    """Per-query recall@k of found against the exact top-k."""
    nq = len(truth_cnt)
    r = np.ones(nq)
    for i in range(nq):
        t = truth_ids[i, :min(k, int(truth_cnt[i]))]
        if len(t) == 0:
            continue
        f = found_ids[i, :min(k, int(found_cnt[i]))]
        r[i] = np.isin(t, f).sum() / len(t)
    return r


def label_actions(recall: np.ndarray, graph_ms: np.ndarray, scan_ms: float,
                  target: float = 1.0) -> np.ndarray:
    """recall [nq][4], graph_ms [nq][4] (per-query graph latency at each ef)
    -> action per query: the fastest graph action whose recall reaches the
    target and whose latency is below the scan's, else scan (0)."""
    nq = recall.shape[0]
    lab = np.zeros(nq, np.int32)
    for i in range(nq):
        best = scan_ms
        for e in range(len(EFS)):
            if recall[i, e] >= target and graph_ms[i, e] < best:
                best = graph_ms[i, e]
                lab[i] = e + 1
    return lab


def routed_batch(index, router: Optional[Router], queries: np.ndarray, preds, k, entries,
                 topb: Optional[int] = None, plan: Optional[np.ndarray] = None,
                 margin: float = 0.0, bp: Optional[BatchPred] = None, split: bool = False):
    """pv_routed_batch -> (ids u64 [nq][topb], dists, cnt, decided ef per query,
    executed (0 answered by the scan / 1 all graph / 2 split), stage_ms [3]: bitmaps, routing (beside the
    search), search; the batch took stage_ms[0] + stage_ms[2]). bp: the
    batch's predicate arrays with entries, if already built. split: each
    query takes its own route even when the batch is scanned."""
    from .pred import concat
    L = _lib.lib()
    q = np.ascontiguousarray(queries, np.float32)
    nq = q.shape[0]
    kk = np.ascontiguousarray(np.broadcast_to(np.asarray(k, np.uint32), (nq,)))
    topb = int(kk.max()) if topb is None else int(topb)
    if bp is None:
        bp = concat(preds, index.count, entries=entries)
    pl = None if plan is None else np.ascontiguousarray(plan, np.uint16)
    out = np.zeros(nq * topb, _lib.HIT_DTYPE)
    cnt = np.zeros(nq, np.uint32)
    dec = np.zeros(nq, np.uint16)
    ex = C.c_int()
    st = np.zeros(3, np.float32)
    err = _err()
    rc = L.pv_routed_batch(index.handle, router._h if router is not None else None, nq, ptr(q),
                           ptr(bp.qd), ptr(bp.nodes), len(bp.nodes), ptr(bp.children),
                           len(bp.children), ptr(bp.invals), len(bp.invals), ptr(kk), topb,
                           ptr(pl), margin, int(split), ptr(out), ptr(cnt), ptr(dec), C.byref(ex),
                           ptr(st),
                           err, len(err))
    if rc != 0:
        raise RuntimeError(err.value.decode())
    out = out.reshape(nq, topb)
    return out["node"], out["dist"], cnt, dec, int(ex.value), st


def feedback_from_batches(samples) -> Feedback:
    """The worker's feedback after homogeneous batches (worker.c:296-333
    attribution: with equal weights in a batch, the per-request sample is
    the batch time). samples: iterable of (graph?, selectivity, batch_ms, n)."""
    fb = Feedback.empty()
    for graph, sel, ms, n in samples:
        si = 1 if graph else 0
        b = sel_bucket(int(sel * 1000))
        us = max(1, int(ms * 1000))
        for arr, idx, val, alpha in ((fb.q_us[si], b, us, n / (n + 64.0)),
                                     (fb.batch_us, si, us, 0.125),
                                     (fb.batch_n16, si, int(n * 16), 0.125)):
            old = int(arr[idx])
            arr[idx] = max(1, val if old == 0 else int(old + alpha * (val - old)))
    return fb


def plain_plan(sel: np.ndarray, k, fb: Optional[Feedback] = None) -> np.ndarray:
    """plain_rule as a pv_routed_batch plan: 0 = scan, else the beam width."""
    graph, ef = plain_rule(sel, np.broadcast_to(np.asarray(k), np.shape(sel)), fb)
    return np.where(graph, np.minimum(ef, 512), 0).astype(np.uint16)
