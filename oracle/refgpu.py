"""The reference's own GPU batch path, timed on this machine's GPU.

Baseline infrastructure (never the measured product): loads
oracle/_ref/libpaves_ref_gpu.so, the reference engine (engine.cpp -DFV_GPU)
linked with the reference's CUDA backend (gpu_engine.cu) compiled for
sm_100a from its own sources, and drives it the way the reference's
PG-free operator microbenchmark does (tools/gpu_micro.cpp:69-206):
fv_index_open -> fv_engine_gpu_precision -> fv_index_gpu_ensure ->
fv_pred_compile / fv_pred_serialize per filter -> back-to-back
fv_gpu_exec_brute_batch / fv_gpu_exec_graph_batch calls with host buffers
(each call is synchronous: H2D, kernels, D2H).

Run as a subprocess (so the reference's CUDA backend and this library never
share a process):

  python -m oracle.refgpu brute --index I --queries Q.npy --classes C.json \
      --batch 64 --topb 10 --precision 0 --steps 60 --out ids.npz
  python -m oracle.refgpu graph --index I --queries Q.npy --classes C.json \
      --batch 64 --k 10 --ef 32,64,128,256 --steps 10 --out ids.npz

C.json: a list of [name, serialized filter] pairs (paves_b200.pred.to_json);
batch i uses class i % len(C) for every query of the batch (the
"--mixed" flag gives query j of every batch class j % len(C) instead).
One JSON line on stdout: per class, wall-clock queries/s of the calls
(e2e, host buffers) and the kernel time the reference's own phase profiler
reports (FV_GPU_PROF, gpu_engine.cu:105-162: kernel + merge per batch).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys
import time

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _ROOT not in sys.path:
    sys.path.insert(0, _ROOT)

from oracle import refengine  # noqa: E402


def _prof_totals(text):
    """Sums the FVPROF lines of the reference's phase profiler."""
    tot = {"brute": {"batches": 0, "kern_ms": 0.0, "merge_ms": 0.0, "h2d_ms": 0.0,
                     "d2h_ms": 0.0},
           "graph": {"batches": 0, "kern_ms": 0.0, "h2d_ms": 0.0, "d2h_ms": 0.0},
           "span": {"batches": 0, "kern_ms": 0.0}}
    for m in re.finditer(r"FVPROF (\{.*\})", text):
        d = json.loads(m.group(1))
        for part, v in tot.items():
            for k in v:
                v[k] += d.get(part, {}).get(k, 0)
    return tot


class _Profiled:
    """Captures fd 2 (where the reference's profiler writes) into a file."""

    def __init__(self):
        import tempfile
        self.f = tempfile.TemporaryFile("w+b")
        self.saved = os.dup(2)

    def __enter__(self):
        sys.stderr.flush()
        os.dup2(self.f.fileno(), 2)
        return self

    def __exit__(self, *exc):
        sys.stderr.flush()
        os.dup2(self.saved, 2)
        os.close(self.saved)
        self.f.seek(0)
        self.text = self.f.read().decode(errors="replace")
        self.f.close()
        return False


def _setup(args):
    from paves_b200 import pred
    os.environ.setdefault("FV_GPU_PROF", "1")
    R = refengine.RefIndex(args.index, kind=args.kind)
    R.gpu_precision(args.precision)
    q = np.load(args.queries).astype(np.float32)
    with open(args.classes) as f:
        classes = [(name, pred.from_json(p)) for name, p in json.load(f)]
    handles = [R.compile(p) for _, p in classes]
    ser = [R.serialize(h) for h in handles]
    return R, q, classes, handles, ser


def _batches(args, q, classes, ser):
    """(class index or -1 for mixed, queries, FvGpuBatchPred list) per step."""
    nb, nc = args.batch, len(classes)
    out = []
    for i in range(max(nc, 1)):
        rows = (np.arange(nb) + i * nb) % len(q)
        if args.mixed:
            bps = [ser[j % nc][0] for j in range(nb)]
            out.append((-1, q[rows], bps, rows))
        else:
            out.append((i, q[rows], [ser[i][0]] * nb, rows))
    return out


def run_brute(args):
    R, q, classes, handles, ser = _setup(args)
    steps = _batches(args, q, classes, ser)
    chunk = min(args.batch, 1024)  # FV_GPU_MAX_BATCH (gpu_engine.h:44)

    def call(qs, bps):
        res = []
        for s in range(0, len(qs), chunk):
            res.append(R.gpu_brute_batch(qs[s:s + chunk], bps[s:s + chunk], args.topb))
        return [np.concatenate(x) for x in zip(*res)]

    for i in range(max(3, args.warmup)):
        _, qs, bps, _ = steps[i % len(steps)]
        call(qs, bps)
    time.sleep(1.1)
    with _Profiled():  # flushes the warm-up's profile
        call(steps[0][1], steps[0][2])
    per = {}
    saved = {}
    with _Profiled() as pr:
        wall = {}
        n = {}
        for i in range(args.steps):
            c, qs, bps, rows = steps[i % len(steps)]
            t0 = time.perf_counter()
            ids, dists, cnt, tr = call(qs, bps)
            dt = time.perf_counter() - t0
            wall[c] = wall.get(c, 0.0) + dt
            n[c] = n.get(c, 0) + 1
            saved[c] = (ids, dists, cnt, rows)
        time.sleep(1.1)
        call(steps[0][1], steps[0][2])  # makes the profiler write its last line
    prof = _prof_totals(pr.text)
    for c in sorted(wall):
        name = classes[c][0] if c >= 0 else "mixed"
        per[name] = {"qps": round(args.batch * n[c] / wall[c], 1),
                     "ms_per_batch": round(1e3 * wall[c] / n[c], 4)}
    tot_wall = sum(wall.values())
    nb_prof = prof["brute"]["batches"] + prof["span"]["batches"]
    kern = prof["brute"]["kern_ms"] + prof["brute"]["merge_ms"] + prof["span"]["kern_ms"]
    line = {"impl": "reference-gpu", "precision": args.precision, "batch": args.batch,
            "topb": args.topb, "steps": args.steps,
            "qps_e2e": round(args.batch * args.steps / tot_wall, 1),
            "classes": per,
            "kernel_ms_per_call": round(kern / max(1, nb_prof), 4) if nb_prof else None,
            "profiled_calls": nb_prof}
    if args.out:
        arrs = {}
        for c, (ids, dists, cnt, rows) in saved.items():
            arrs.update({f"ids_{c}": ids, f"dists_{c}": dists, f"cnt_{c}": cnt,
                         f"rows_{c}": rows})
        np.savez(args.out, **arrs)
    print(json.dumps(line), flush=True)
    for h in handles:
        R.free_pred(h)
    R.close()


def run_graph(args):
    R, q, classes, handles, ser = _setup(args)
    nb = args.batch
    qs = q[:nb]
    entries = np.array([R.graph_entry(x) for x in qs], np.uint32)
    res = []
    out = {}
    for c, (name, _) in enumerate(classes):
        bps = [ser[c][0]] * nb
        for ef in [int(x) for x in args.ef.split(",")]:
            mv = max(200000, 400 * ef)  # exec.c:289-290
            for _ in range(max(1, args.warmup)):
                R.gpu_graph_batch(qs, entries, bps, ef, mv)
            t0 = time.perf_counter()
            for _ in range(args.steps):
                ids, dists, cnt, ex = R.gpu_graph_batch(qs, entries, bps, ef, mv)
            dt = time.perf_counter() - t0
            res.append({"filter": name, "ef": ef, "qps": round(nb * args.steps / dt, 1)})
            out[f"{name}_{ef}_ids"] = ids[:, :args.k]
            out[f"{name}_{ef}_cnt"] = np.minimum(cnt, args.k)
    if args.out:
        np.savez(args.out, **out)
    print(json.dumps({"impl": "reference-gpu", "precision": args.precision, "batch": nb,
                      "results": res}), flush=True)
    for h in handles:
        R.free_pred(h)
    R.close()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["brute", "graph"])
    ap.add_argument("--index", required=True)
    ap.add_argument("--queries", required=True)
    ap.add_argument("--classes", required=True)
    ap.add_argument("--kind", default="gpu", choices=["gpu", "dropin"])
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--topb", type=int, default=10)
    ap.add_argument("--k", type=int, default=10)
    ap.add_argument("--ef", default="32,64,128,256")
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    (run_brute if args.mode == "brute" else run_graph)(args)


if __name__ == "__main__":
    main()
