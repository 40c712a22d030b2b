"""What the trained router gains over the method without it.

The router is trained here, on the GPU, from labels the method generates
(paves_b200.router_train: every training query runs the scan and the graph
search at each ef). Six held-out batches (one per filter class, 64 queries,
top-10) then run through pv_routed_batch three ways:

  learned      the MLP's action per query
  plain        the reference's rule without feedback (planner.c seeds:
               graph 0.5 ms < scan 1.0 ms, so the graph at exec.c's ef)
  plain+fb     the same rule after the worker's feedback from running
               every class both ways

and the test reports recall@10 per class and device time per batch. The
bar: the learned router reaches recall@10 >= 0.95 in every class, never
has a lower worst-class recall than the plain rule, takes less device
time over the six classes than the plain rule (the gain over the rule it
replaces: on this index the graph search at the rule's beam widths is the
slower path for every class, which the labels teach the router), and is
not slower than the plain rule with feedback beyond its own routing cost.
"""
import json

import numpy as np
import pytest

from paves_b200 import GpuIndex, _lib, datagen, pred
from paves_b200.hnsw import Hnsw
from paves_b200.router import (Router, feedback_from_batches, init_params, kmeans,
                               plain_plan, routed_batch)
from paves_b200.router_train import KS, calibrate, label_queries, random_predicates, \
    standardization

pytestmark = pytest.mark.gpu
N, D, NTRAIN, NQ, K = 200_000, 128, 16384, 64, 10


def _recall(ids, cnt, truth, tcnt):
    r = []
    for i in range(len(cnt)):
        t = truth[i, :min(K, int(tcnt[i]))]
        if len(t) == 0:
            r.append(1.0)
            continue
        r.append(np.isin(t, ids[i, :int(cnt[i])]).sum() / len(t))
    return float(np.mean(r))


def test_learned_router_vs_plain_rule():
    ds = datagen.make_dataset(N, D, nq=16)
    h = Hnsw(ds.vectors, 16, 100)
    g = GpuIndex(ds.vectors, ds.cols, l0=h.l0, precision=_lib.FV_GPU_PREC_BF16)
    r = Router(kmeans(ds.vectors, 256, iters=6, sample=65536))
    rng = np.random.default_rng(datagen.SEED + 5)
    tq = datagen.make_queries(ds.centers, NTRAIN, stream=5)
    tp = random_predicates(rng, NTRAIN)
    tk = rng.choice(np.asarray(KS, np.uint32), NTRAIN)
    scan_ms, step_ms = calibrate(g, h.entries, tq, tp)
    feats, labels, _, _ = label_queries(g, h.entries, r, tq, tp, tk, scan_ms, step_ms)
    mean, std = standardization(feats)
    r.set_params(init_params(1), mean, std)
    hist = r.train(feats, labels, epochs=20, batch=1024, lr=3e-3)
    assert hist[-1] < hist[0]

    classes = datagen.six_predicates()
    eq = datagen.make_queries(ds.centers, NQ * len(classes), stream=2)
    report, samples, per = {}, [], {}
    for ci, (name, p) in enumerate(classes.items()):
        q = eq[ci * NQ:(ci + 1) * NQ]
        ent = h.entries(q)
        preds = [p] * NQ
        sel = float(pred.eval_numpy(p, ds.cols).mean())
        # exact truth: the scan (exact on this integer data)
        ti, _, tc, _, _, st_scan = routed_batch(g, None, q, preds, K, ent,
                                                plan=np.zeros(NQ, np.uint16))
        cold = plain_plan(np.full(NQ, sel), K)
        gi, _, gc, _, ex_g, st_graph = routed_batch(g, None, q, preds, K, ent, plan=cold)
        samples += [(False, sel, float(st_scan[0] + st_scan[2]), NQ),
                    (True, sel, float(st_graph[0] + st_graph[2]), NQ)]
        per[name] = (q, ent, preds, sel, ti, tc, cold, (gi, gc, st_graph))
    fb = feedback_from_batches(samples)
    for name, (q, ent, preds, sel, ti, tc, cold, (gi, gc, st_cold)) in per.items():
        li, _, lc, dec, ex_l, st_l = routed_batch(g, r, q, preds, K, ent)
        warm = plain_plan(np.full(NQ, sel), K, fb)
        wi, _, wc, _, ex_w, st_w = routed_batch(g, None, q, preds, K, ent, plan=warm)
        report[name] = {
            "learned": {"recall": _recall(li, lc, ti, tc), "ms": float(st_l[0] + st_l[2]),
                        "graph": ex_l, "graph_frac": float((dec > 0).mean())},
            "plain": {"recall": _recall(gi, gc, ti, tc), "ms": float(st_cold[0] + st_cold[2]),
                      "ef": int(cold[0])},
            "plain_fb": {"recall": _recall(wi, wc, ti, tc), "ms": float(st_w[0] + st_w[2]),
                         "ef": int(warm[0])},
        }
    print(json.dumps({"scan_ms": scan_ms, "step_ms": step_ms,
                      "labels": np.bincount(labels, minlength=5).tolist(), "classes": report}))
    lr = [v["learned"]["recall"] for v in report.values()]
    pr = [v["plain"]["recall"] for v in report.values()]
    assert min(lr) >= 0.95, report
    assert min(lr) >= min(pr) - 1e-9, report
    t_learned = sum(v["learned"]["ms"] for v in report.values())
    t_plain = sum(v["plain"]["ms"] for v in report.values())
    t_fb = sum(v["plain_fb"]["ms"] for v in report.values())
    assert t_learned < t_plain, report
    # the learned path pays features + MLP beside its speculative scan
    assert t_learned <= 1.25 * t_fb + 0.05 * len(report), report
    r.close()
    g.close()
