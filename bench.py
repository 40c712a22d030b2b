#!/usr/bin/env python
"""Benchmark of the PAVES GPU search path on B200.

Workload (synthetic, seeded; stands in for SIFT1M): N = 1,000,000 rows x
128 dims from the Gaussian-mixture generator, two attribute columns, an
HNSW graph (M=16, efConstruction=200) built by the library, and six
batches of 64 queries, one per filter class (0.1% .. 95% selectivity),
filtered L2 top-10. A step is one batch; steps rotate through the classes.

  value     chosen path: the learned router (features + MLP on the device)
            sends each batch to the BF16 tensor-core scan + exact FP32
            re-rank, or to the graph search at a per-query beam width
            (pv_routed_batch); queries/s over the device time of K steps
            (bitmaps, routing, search), max over ranks
  plain_gpu exact FP32 answers for the same batches (prepared, resident):
            the f32 rows read as TF32 on the tensor cores with a certified
            exact re-rank, and (cuda_cores_only) the CUDA-core scan
  e2e       the chosen path through the C ABI with host buffers: predicate
            compile + H2D + kernels + D2H, wall clock
  roofline  the tensor-core scan kernel: algorithmic bytes (rows once per
            batch) over its average CUDA-event duration, against
            MEASURED_PEAKS.json
  cpu_baseline  the reference engine's CPU BruteCursor (oracle/_ref, built
            from the reference sources) over the 384 queries, all host
            cores, after one warm-up pass (the method --impl reference
            repeats per step)
  parity_vs_reference_cpu  that run's answers against the plain exact
            path's and the chosen path's: queries with identical ids and
            identical FP32 distances, at 1M rows
  reference_gpu  the reference's own CUDA backend (gpu_engine.cu built for
            sm_100a, oracle/_ref) on the same index, batches and filters,
            fp32 and sq8, through the engine's batch call with host buffers
            (a subprocess): e2e queries/s, its profiler's kernel time, and
            its answers against the reference CPU's
  graph_search_points  the graph search alone on the same index's graph:
            filters at 1 %, 10 %, 50 %, ef 32..256, recall@10 and queries/s
  uneven_microbatches  100 micro-batches over 10M x 96 FP8 rows (sizes
            1..512, per-query k and filter) through the CUDA-graph executor
            and through the persistent kernel: p50/p99 latency, queries/s
  (--no-extras skips the last two)

--impl reference times that reference CPU path alone (rank 0).
Multi-GPU (torchrun): each rank serves its own batches on its own GPU
(independent replicas, weak scaling; the scan needs no collective).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from paves_b200 import _lib, datagen, pred  # noqa: E402
from paves_b200.index import GpuIndex  # noqa: E402

METRIC = "filtered top-10 QPS, 1M x 128 L2"
N_ROWS, DIM, BATCH, TOPK = 1_000_000, 128, 64, 10


def load_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu capture
    summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return int(json.load(f)[kernel]["bytes_per_launch"])
    except Exception:
        return None


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={device}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.p is None:
            return out
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows]
        mx = [float(r[2]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for i, nme in enumerate(names):
                if r[5 + i].strip().lower() == "active":
                    reasons.add(nme)
        out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), reasons=sorted(reasons),
                   samples=len(rows))
        return out


def make_workload(n=N_ROWS, d=DIM, nb=BATCH):
    """Data set and the six filter classes; class c owns queries
    [c * nb, (c + 1) * nb). Returns (ds, classes [(name, pred)], preds per query)."""
    classes = list(datagen.six_predicates().items())
    ds = datagen.make_dataset(n, d, nq=nb * len(classes))
    preds = [classes[q // nb][1] for q in range(nb * len(classes))]
    return ds, classes, preds


ROUTER_FILE = os.path.join(ROOT, "paves_b200", "router_1m128.npz")


# ---------------------------------------------------------------- reference CPU
def write_brute_index(ds, path):
    """The rows and attribute columns as a PAVES index file (a one-neighbour
    level 0: the brute paths read no graph)."""
    from paves_b200.indexfile import write_index
    n = ds.vectors.shape[0]
    l0 = np.zeros((n, 3), np.uint32)
    write_index(path, ds.vectors, ds.cols, 1, 1, np.zeros(n, np.uint8), l0,
                np.zeros(n + 1, np.uint64), np.zeros(0, np.uint32), 0, 0)


def reference_cpu_qps(path, ds, preds, budget_s=20.0, threads=None, keep=False):
    """Reference engine BruteCursor (built from the reference sources), one
    query at a time with `threads` workers, over up to len(preds) queries
    within budget_s. Returns (qps, queries_run, threads, answers) with
    answers[q] = (ids, dists) when keep."""
    from oracle import refengine
    threads = threads or os.cpu_count() or 1
    R = refengine.RefIndex(path)
    handles = {}
    answers = {}
    done = 0
    t0 = time.perf_counter()
    for q, p in enumerate(preds):
        key = id(p)
        if key not in handles:
            handles[key] = R.compile(p)
        res = R.brute(ds.queries[q], handles[key], TOPK, threads=threads)
        if keep:
            answers[q] = res
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    for h in handles.values():
        R.free_pred(h)
    R.close()
    return done / dt, done, threads, answers


def reference_cpu_leg(path, ds, preds, warmup, steps, keep=False):
    """The CPU baseline both arms report: `warmup` untimed passes over 8
    queries, then `steps` timed passes over the workload's queries (10 s
    budget each); the median pass. Returns (qps, queries per pass, threads,
    answers of the last pass)."""
    for _ in range(warmup):
        reference_cpu_qps(path, ds, preds[:8], budget_s=5.0)
    per, ans, nrun, threads = [], {}, 0, 1
    for i in range(steps):
        qps, nrun, threads, ans = reference_cpu_qps(path, ds, preds, budget_s=10.0,
                                                    keep=keep and i == steps - 1)
        per.append(qps)
    return float(np.median(per)), nrun, threads, ans


def run_reference(args, rank, world):
    if rank != 0:
        return
    ds, _, preds = make_workload()
    with tempfile.TemporaryDirectory(dir="/tmp") as td:
        path = os.path.join(td, "bench.idx")
        write_brute_index(ds, path)
        qps, nrun, threads, _ = reference_cpu_leg(path, ds, preds, args.warmup, args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(qps, 2), "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * BATCH / qps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "1M x 128 Gaussian-mixture rows, 64-query batches, six "
                               "predicate classes, top-10, reference CPU BruteCursor",
                   "rows": N_ROWS, "dim": DIM, "batch": BATCH, "k": TOPK},
        "cpu_baseline": {"value": round(qps, 2), "unit": "queries/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{nrun} queries (the six class batches) per step, one at "
                                   "a time; median of the steps"},
        "e2e": {"value": round(qps, 2), "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_gpu_leg(path, ds, classes, steps, precisions=(0, 1), timeout=600):
    """The reference's own CUDA backend (gpu_engine.cu built for sm_100a,
    oracle/_ref/libpaves_ref_gpu.so) on the same index, batches and filters,
    through the engine's batch call with host buffers, in a subprocess
    (oracle/refgpu.py). Per precision (0 = fp32 exact, 1 = sq8): e2e
    queries/s, the kernel time its own profiler reports, and the answers."""
    from oracle import refengine
    if not refengine.available("gpu"):
        return {"unavailable": "oracle/_ref/libpaves_ref_gpu.so not built"}, {}
    td = os.path.dirname(path)
    qf = os.path.join(td, "queries.npy")
    cf = os.path.join(td, "classes.json")
    np.save(qf, ds.queries[:BATCH * len(classes)])
    with open(cf, "w") as f:
        json.dump([[n, pred.to_json(p)] for n, p in classes], f)
    out, answers = {}, {}
    for prec in precisions:
        name = {0: "fp32", 1: "sq8"}[prec]
        of = os.path.join(td, f"ref_{name}.npz")
        cmd = [sys.executable, "-m", "oracle.refgpu", "brute", "--index", path, "--queries", qf,
               "--classes", cf, "--batch", str(BATCH), "--topb", str(TOPK), "--precision",
               str(prec), "--steps", str(max(steps, len(classes))), "--out", of]
        try:
            r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=timeout)
            if r.returncode != 0:
                out[name] = {"failed": (r.stderr or r.stdout).strip().splitlines()[-1:]}
                continue
            out[name] = json.loads(r.stdout.strip().splitlines()[-1])
            z = np.load(of)
            answers[name] = {int(k.split("_")[1]): (z[k], z[f"cnt_{k.split('_')[1]}"])
                             for k in z.files if k.startswith("ids_")}
        except Exception as e:  # informative only
            out[name] = {"failed": str(e)}
    return out, answers


# ---------------------------------------------------------------- ours
def prepared_batch(gi, queries, bp, topb, mode):
    L = _lib.lib()
    err = C.create_string_buffer(512)
    q = np.ascontiguousarray(queries, np.float32)
    b = L.pv_batch_create(gi.handle, q.shape[0], _lib.ptr(q), _lib.ptr(bp.qd),
                          _lib.ptr(bp.nodes), len(bp.nodes), _lib.ptr(bp.children),
                          len(bp.children), _lib.ptr(bp.invals), len(bp.invals), topb, mode,
                          err, 512)
    if not b:
        raise RuntimeError(err.value.decode())
    return b


def batch_run(b, iters, stages=False):
    L = _lib.lib()
    err = C.create_string_buffer(512)
    st = (C.c_float * 4)()
    tot = C.c_float()
    rc = L.pv_batch_run(b, iters, st if stages else None, C.byref(tot), err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return tot.value, list(st)


def fetch(b, nq, topb):
    L = _lib.lib()
    err = C.create_string_buffer(512)
    out = np.zeros(nq * topb, _lib.HIT_DTYPE)
    cnt = np.zeros(nq, np.uint32)
    tr = np.zeros(nq, np.uint8)
    if L.pv_batch_fetch(b, _lib.ptr(out), _lib.ptr(cnt), _lib.ptr(tr), err, 512) != 0:
        raise RuntimeError(err.value.decode())
    out = out.reshape(nq, topb)
    return out["node"], out["dist"], cnt, tr


KERNEL_CASES = {
    # name: (batch, precision, mode, predicate kind index or None for rotation)
    "exact_b1": (1, _lib.FV_GPU_PREC_FP32, _lib.PV_MODE_EXACT, 5),
    "exact_b64": (64, _lib.FV_GPU_PREC_FP32, _lib.PV_MODE_EXACT, None),
    # the same on the CUDA cores alone (pv_exact_tc off)
    "exact_b64_cuda": (64, _lib.FV_GPU_PREC_FP32, _lib.PV_MODE_EXACT, None),
    "bf16_b64": (64, _lib.FV_GPU_PREC_BF16, _lib.PV_MODE_LOW, None),
    # one selective class per batch: the sparse route (0.1 %, 1 %)
    "bf16_b64_sel01": (64, _lib.FV_GPU_PREC_BF16, _lib.PV_MODE_LOW, 0),
    "bf16_b64_sel1": (64, _lib.FV_GPU_PREC_BF16, _lib.PV_MODE_LOW, 1),
    "fp8_b64": (64, _lib.FV_GPU_PREC_FP8, _lib.PV_MODE_LOW, None),
    # one dense class per batch, as the headline's class batches (10 %, 95 %)
    "bf16_b64_sel10": (64, _lib.FV_GPU_PREC_BF16, _lib.PV_MODE_LOW, 2),
    "bf16_b64_sel95": (64, _lib.FV_GPU_PREC_BF16, _lib.PV_MODE_LOW, 5),
    "exact_b64_sel10": (64, _lib.FV_GPU_PREC_FP32, _lib.PV_MODE_EXACT, 2),
    # graph: 200k x 128 rows, HNSW M=16 efC=100, 64 queries, 10% filter, ef 64
    "graph_b64": (64, None, None, None),
}


def kernel_case(name, iters, tc_shape=None):
    """One batch shape run `iters` times after 3 warm-up runs (device-
    resident inputs): the small, self-contained program that ncu captures
    profile. tc_shape = (epi, stages, grow, replicas, seed), 0 = automatic."""
    nq, prec, mode, pk = KERNEL_CASES[name]
    if name == "graph_b64":
        from paves_b200.hnsw import Hnsw
        ds = datagen.make_dataset(200_000, DIM, nq=nq)
        h = Hnsw(ds.vectors, 16, 100)
        gi = GpuIndex(ds.vectors, ds.cols, l0=h.l0)
        p = datagen.graph_predicates()["sel10%"]
        ent = h.entries(ds.queries)
        ms = 0.0
        for _ in range(iters):
            gi.graph_batch(ds.queries, ent, [p] * nq, 64)
            ms += _lib.lib().pv_last_kernel_ms(gi.handle)
        print(json.dumps({"case": name, "iters": iters, "ms": round(ms / iters, 4)}))
        gi.close()
        return
    ds, classes, _ = make_workload(nb=max(nq, 1))
    if pk is not None:
        preds = [classes[pk][1]] * nq
    else:
        preds = [classes[q % len(classes)][1] for q in range(nq)]
    gi = GpuIndex(ds.vectors, ds.cols, precision=prec)
    if name.endswith("_cuda"):
        _lib.lib().pv_exact_tc(gi.handle, 0)
    if tc_shape:
        if _lib.lib().pv_tc_shape(gi.handle, *tc_shape) != 0:
            raise ValueError(f"bad tensor-core shape {tc_shape}")
    bp = pred.concat(preds[:nq], N_ROWS)
    b = prepared_batch(gi, ds.queries[:nq], bp, TOPK, mode)
    batch_run(b, 3)
    _, st = batch_run(b, iters, stages=True)
    # the stages are timed apart (an event between them stops the kernels of
    # one stage from starting under the last kernel of the one before);
    # total_ms is the same batch without them
    tot, _ = batch_run(b, iters)
    print(json.dumps({"case": name, "iters": iters, "total_ms": round(tot / iters, 4),
                      "stage_ms": [round(x / iters, 4) for x in st]}))
    _lib.lib().pv_batch_free(b)
    gi.close()


def stream_filter(rng):
    """A per-query filter of selectivity log-uniform in 0.05%..90%: a price
    range, AND a category set (5 of 10) for a third of the queries."""
    P, Cc = datagen.COL_PRICE, datagen.COL_CATEGORY
    sel = float(np.exp(rng.uniform(np.log(0.0005), np.log(0.9))))
    cat = rng.random() < 1 / 3
    width = 1000.0 * min(1.0, sel * (2.0 if cat else 1.0))
    a = float(rng.uniform(0, 1000.0 - width))
    p = pred.And(pred.Cmp(P, ">=", a), pred.Cmp(P, "<", a + width))
    if cat:
        p = pred.And(p, pred.In(Cc, [float(c) for c in sorted(rng.choice(10, 5, replace=False))]))
    return p


def stream_bench(args):
    """Uneven micro-batches: N = 10M x 96 (256-component mixture), FP8
    per-row-scaled tensor-core scan + exact FP32 re-rank, sizes log-uniform
    in 1..512, k from {1, 10, 100} and a filter per query. The same
    sequence of batches runs twice: through the stream's autotuned CUDA
    graphs (paves_b200.stream.Stream, one graph replay per batch) and
    through the persistent kernel (paves_b200.stream.Serve, one resident
    kernel consuming the queue). One micro-batch per step; latency = host
    wall time of the call; device time = the graph's CUDA-event time, or
    the persistent kernel's GPU-clock time from taking the batch to its
    completion word."""
    res = stream_results(args.steps, args.warmup)
    line = {
        "metric": "uneven micro-batch QPS, 10M x 96 L2, FP8 + FP32 re-rank",
        "value": res["graphs"]["value"], "unit": "queries/s", "n_gpus": 1,
        "steps": args.steps, "higher_is_better": True, "dtype": "fp8-e4m3", "data": "synthetic",
        "config": STREAM_CONFIG,
    }
    line.update({k: v for k, v in res["graphs"].items() if k != "value"})
    line["persistent_kernel"] = res["persistent_kernel"]
    print(json.dumps(line), flush=True)


STREAM_CONFIG = {"workload": "10M x 96 Gaussian-mixture rows (256 components); micro-batch "
                             "sizes log-uniform 1..512; k in {1, 10, 100} and a filter "
                             "(selectivity log-uniform 0.05%-90%) per query",
                 "rows": 10_000_000, "dim": 96, "max_batch": 512, "max_k": 100,
                 "executor": "CUDA graph per batch-size bucket (value); persistent kernel "
                             "beside it"}


def stream_results(nsteps, nwarm):
    """The measurement behind stream_bench: {"graphs": ..., "persistent_kernel": ...}."""
    from paves_b200.stream import Serve, Stream
    n, d = 10_000_000, 96
    ds = datagen.make_dataset(n, d, nq=1024, ncomp=256)
    gi = GpuIndex(ds.vectors, ds.cols, precision=_lib.FV_GPU_PREC_FP8)
    tune = os.path.join(tempfile.gettempdir(), f"paves_stream_tune_{n}x{d}.txt")
    rng = np.random.default_rng(datagen.SEED + 9)

    def batch():
        nq = int(np.clip(np.exp(rng.uniform(0, np.log(512))), 1, 512))
        idx = rng.integers(0, ds.queries.shape[0], nq)
        k = rng.choice(np.array([1, 10, 100], np.uint32), nq)
        return ds.queries[idx], [stream_filter(rng) for _ in range(nq)], k

    warm = [batch() for _ in range(max(3, nwarm))]
    steps = [batch() for _ in range(nsteps)]
    truth = {}
    for i in range(0, nsteps, 10):  # the exact FP32 scan of every 10th batch
        q, preds, k = steps[i]
        bx = prepared_batch(gi, q, pred.concat(preds, n), 100, _lib.PV_MODE_EXACT)
        batch_run(bx, 1)
        xi, _, xc, _ = fetch(bx, len(q), 100)
        _lib.lib().pv_batch_free(bx)
        truth[i] = (xi, xc)

    def measure(runner):
        for q, preds, k in warm:
            runner(q, preds, k)
        lat, dev, nqs, recs = [], [], [], []
        clk = Clocks(0)
        for i, (q, preds, k) in enumerate(steps):
            t = time.perf_counter()
            ids, _, cnt, ms = runner(q, preds, k)
            lat.append((time.perf_counter() - t) * 1e3)
            dev.append(ms)
            nqs.append(len(q))
            if i in truth:
                xi, xc = truth[i]
                for j in range(len(q)):
                    t_ids = xi[j, :min(int(k[j]), int(xc[j]))]
                    if len(t_ids):
                        recs.append(np.isin(t_ids, ids[j, :cnt[j]]).mean())
        clocks = clk.stop()
        lat = np.asarray(lat)
        return {"value": round(sum(nqs) / (sum(dev) / 1e3), 1),
                "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                               "p99": round(float(np.percentile(lat, 99)), 3),
                               "mean": round(float(lat.mean()), 3)},
                "device_ms": {"p50": round(float(np.percentile(dev, 50)), 3),
                              "p99": round(float(np.percentile(dev, 99)), 3)},
                "e2e": {"value": round(sum(nqs) / (lat.sum() / 1e3), 1), "unit": "queries/s"},
                "recall_vs_exact": round(float(np.mean(recs)), 4) if recs else None,
                "queries": int(sum(nqs)), "clocks": clocks}

    t0 = time.perf_counter()
    s = Stream(gi, 512, 100, ds.queries[:512], tune)
    setup_s = time.perf_counter() - t0
    graphs = measure(s.run)
    graphs["setup_s"] = round(setup_s, 1)
    graphs["plans"] = s.plans()
    s.close()
    persistent = None
    try:
        sv = Serve(gi, 512, 100, idle_ms=1000)
        persistent = measure(sv.run)
        persistent["status"] = sv.status()
        sv.close()
    except Exception as e:  # reported, the graph executor's line stands
        persistent = {"failed": str(e)}
    gi.close()
    return {"graphs": graphs, "persistent_kernel": persistent}


def graph_points(gi, q, ent, steps, warmup):
    """Config 3's points on gi's graph: filters at 1 %, 10 % and 50 %, ef 32 to
    256, 64-query batches; recall@10 against the exact scan, device-time
    and wall-clock queries/s, mean steps and visited nodes per query."""
    L = _lib.lib()
    args = argparse.Namespace(steps=steps, warmup=warmup)
    res = []
    for name, p in datagen.graph_predicates().items():
        preds = [p] * BATCH
        xi, _, xc, _ = gi.brute_batch(q, preds, TOPK)
        for ef in (32, 64, 128, 256):
            for _ in range(max(1, args.warmup)):
                gi.graph_batch(q, ent, preds, ef)
            dev = 0.0
            reps = max(1, min(args.steps, 10))
            t0 = time.perf_counter()
            for _ in range(reps):
                ids, _, cnt, _ = gi.graph_batch(q, ent, preds, ef)
                dev += L.pv_last_kernel_ms(gi.handle)
            wall = time.perf_counter() - t0
            rec = float(np.mean([np.isin(xi[i, :xc[i]], ids[i, :TOPK]).sum() / max(1, int(xc[i]))
                                 for i in range(BATCH)]))
            st = np.zeros(BATCH * 4, np.uint32)
            L.pv_graph_stats(gi.handle, _lib.ptr(st), BATCH)
            st = st.reshape(BATCH, 4)
            res.append({"filter": name, "ef": ef, "recall_at_10": round(rec, 4),
                        "qps": round(BATCH * reps / (dev / 1e3), 1),
                        "qps_e2e": round(BATCH * reps / wall, 1),
                        "mean_steps": round(float(st[:, 0].mean()), 1),
                        "mean_visited": round(float(st[:, 1].mean()), 1)})
    return res


def graph_bench(args):
    """Filtered graph search: the 1M x 128 set, HNSW (M=16, efConstruction
    200) built by the library, 64 queries per batch, filters at 1%, 10% and
    50%, ef in {32, 64, 128, 256}; recall@10 against the exact scan and
    device-time and wall-clock (host buffers) QPS, beside the reference
    engine's HnswCursor (built from its sources) on the same graph file, one
    query per host thread, and the reference's own GPU graph kernel through
    the engine's batch call (wall clock, host buffers)."""
    from concurrent.futures import ThreadPoolExecutor
    ds, _, _ = make_workload()
    cache = os.path.join(tempfile.gettempdir(), f"paves_bench_hnsw_{N_ROWS}x{DIM}.npz")
    t0 = time.perf_counter()
    h = shared_graph(ds.vectors, 0, None, cache)
    build_s = time.perf_counter() - t0
    gi = GpuIndex(ds.vectors, ds.cols, l0=h.l0)
    L = _lib.lib()
    q = ds.queries[:BATCH]
    ent = h.entries(q)
    res = graph_points(gi, q, ent, args.steps, args.warmup)
    # the same searches on the graph the GPU builder makes (pv_hnsw_build_gpu)
    gpu_built = {}
    try:
        from paves_b200.hnsw import Hnsw
        t0 = time.perf_counter()
        hg = Hnsw(ds.vectors, 16, builder="gpu")
        gpu_built["build_s"] = round(time.perf_counter() - t0, 2)
        gg = GpuIndex(ds.vectors, ds.cols, l0=hg.l0)
        entg = hg.entries(q)
        rows = []
        for name, p in datagen.graph_predicates().items():
            preds = [p] * BATCH
            xi, _, xc, _ = gi.brute_batch(q, preds, TOPK)
            for ef in (32, 64, 128, 256):
                gg.graph_batch(q, entg, preds, ef)
                dev = 0.0
                reps = max(1, min(args.steps, 10))
                for _ in range(reps):
                    ids, _, cnt, _ = gg.graph_batch(q, entg, preds, ef)
                    dev += L.pv_last_kernel_ms(gg.handle)
                rec = float(np.mean([np.isin(xi[i, :xc[i]], ids[i, :TOPK]).sum() /
                                     max(1, int(xc[i])) for i in range(BATCH)]))
                rows.append({"filter": name, "ef": ef, "recall_at_10": round(rec, 4),
                             "qps": round(BATCH * reps / (dev / 1e3), 1)})
        gpu_built["results"] = rows
        gg.close()
    except Exception as e:  # informative
        gpu_built = {"failed": str(e)}
    ref = []
    try:
        from oracle import refengine
        if refengine.available("cpu"):
            path = os.path.join(tempfile.gettempdir(), "paves_bench_graph.idx")
            h.write(path, ds.cols)
            R = refengine.RefIndex(path)
            thr = os.cpu_count() or 1
            for name, p in datagen.graph_predicates().items():
                ph = R.compile(p)
                xi, _, xc, _ = gi.brute_batch(q, [p] * BATCH, TOPK)
                for ef in (32, 64, 128, 256):
                    t0 = time.perf_counter()
                    with ThreadPoolExecutor(thr) as ex:
                        outs = list(ex.map(lambda i: R.hnsw(q[i], ph, TOPK, ef)[0], range(BATCH)))
                    wall = time.perf_counter() - t0
                    rec = float(np.mean([np.isin(xi[i, :xc[i]], outs[i]).sum() / max(1, int(xc[i]))
                                         for i in range(BATCH)]))
                    ref.append({"filter": name, "ef": ef, "recall_at_10": round(rec, 4),
                                "qps": round(BATCH / wall, 1), "threads": thr})
                R.free_pred(ph)
            R.close()
    except Exception as e:  # the reference arm is informative only
        ref = [{"failed": str(e)}]
    # the reference's own GPU graph kernel (fv_graph_kernel, gpu_engine.cu
    # built for sm_100a) on the same graph file, entries and filters
    ref_gpu = []
    try:
        from oracle import refengine
        if refengine.available("gpu") and not args.no_ref_gpu:
            td = tempfile.mkdtemp(dir="/tmp")
            path = os.path.join(td, "graph.idx")
            h.write(path, ds.cols)
            qf, cf, of = (os.path.join(td, x) for x in ("q.npy", "c.json", "ids.npz"))
            np.save(qf, q)
            gp = list(datagen.graph_predicates().items())
            with open(cf, "w") as f:
                json.dump([[n, pred.to_json(p)] for n, p in gp], f)
            cmd = [sys.executable, "-m", "oracle.refgpu", "graph", "--index", path, "--queries",
                   qf, "--classes", cf, "--batch", str(BATCH), "--k", str(TOPK), "--ef",
                   "32,64,128,256", "--steps", str(max(1, min(args.steps, 10))), "--out", of]
            r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
            if r.returncode != 0:
                ref_gpu = [{"failed": (r.stderr or r.stdout).strip().splitlines()[-1:]}]
            else:
                rl = json.loads(r.stdout.strip().splitlines()[-1])
                z = np.load(of)
                for e in rl["results"]:
                    p = dict(gp)[e["filter"]]
                    xi, _, xc, _ = gi.brute_batch(q, [p] * BATCH, TOPK)
                    ids = z[f"{e['filter']}_{e['ef']}_ids"]
                    cnt = z[f"{e['filter']}_{e['ef']}_cnt"]
                    e["recall_at_10"] = round(float(np.mean(
                        [np.isin(xi[i, :xc[i]], ids[i, :cnt[i]]).sum() / max(1, int(xc[i]))
                         for i in range(BATCH)])), 4)
                    ref_gpu.append(e)
            for f in (path, qf, cf, of):
                if os.path.exists(f):
                    os.unlink(f)
            os.rmdir(td)
    except Exception as e:
        ref_gpu = [{"failed": str(e)}]
    line = {"metric": "filtered graph search QPS, 1M x 128 L2, HNSW level 0", "unit": "queries/s",
            "value": max(r["qps"] for r in res), "higher_is_better": True, "n_gpus": 1,
            "data": "synthetic",
            "config": {"workload": "1M x 128 Gaussian-mixture rows, HNSW M=16 efC=200 built by "
                                   "the library, 64-query batches, filters 1%/10%/50%, top-10",
                       "rows": N_ROWS, "dim": DIM, "batch": BATCH, "k": TOPK},
            "host_build_s": round(build_s, 1), "results": res, "gpu_built_graph": gpu_built,
            "reference_cpu": ref, "reference_gpu": ref_gpu}
    print(json.dumps(line), flush=True)
    gi.close()


def batches_bench(args):
    """Batch sizes 1, 64, 512 and 4096 on the 1M x 128 set, filters rotating
    per query through the six classes, top-10: this library through
    fv_gpu_brute_batch with host buffers (exact FP32 upload, and BF16 upload
    = tensor-core scan + exact re-rank), calls of at most 1024 queries
    (FV_GPU_MAX_BATCH), wall clock; beside the reference's own CUDA backend
    (oracle/_ref, fp32 and sq8) driven the same way in a subprocess. Also
    this library's device time per batch (prepared, resident inputs)."""
    ds, classes, _ = make_workload(nb=4096 // 6 + 1)
    nq_all = 4096
    preds = [classes[q % len(classes)][1] for q in range(nq_all)]
    sizes = [1, 64, 512, 4096]
    out = {"ours": {}, "reference_gpu": {}}
    reps = {1: 60, 64: 30, 512: 8, 4096: 3}
    for prec, name in ((_lib.FV_GPU_PREC_FP32, "fp32"), (_lib.FV_GPU_PREC_BF16, "bf16")):
        gi = GpuIndex(ds.vectors, ds.cols, precision=prec)
        res = {}
        for B in sizes:
            q = ds.queries[:B]

            def call():
                for s0 in range(0, B, 1024):
                    gi.brute_batch(q[s0:s0 + 1024], preds[s0:min(B, s0 + 1024)], TOPK)

            for _ in range(2):
                call()
            t0 = time.perf_counter()
            for _ in range(reps[B]):
                call()
            wall = (time.perf_counter() - t0) / reps[B]
            bp = pred.concat(preds[:B], N_ROWS)
            b = prepared_batch(gi, q, bp, TOPK, _lib.PV_MODE_EXACT if prec ==
                               _lib.FV_GPU_PREC_FP32 else _lib.PV_MODE_LOW)
            batch_run(b, 2)
            ms, _ = batch_run(b, reps[B])
            _lib.lib().pv_batch_free(b)
            res[str(B)] = {"qps_e2e": round(B / wall, 1), "ms_e2e": round(1e3 * wall, 3),
                           "qps_device": round(B * reps[B] / (ms / 1e3), 1),
                           "ms_device": round(ms / reps[B], 4)}
        out["ours"][name] = res
        gi.close()
    from oracle import refengine
    if refengine.available("gpu") and not args.no_ref_gpu:
        td = tempfile.mkdtemp(dir="/tmp")
        path = os.path.join(td, "b.idx")
        write_brute_index(ds, path)
        qf, cf = os.path.join(td, "q.npy"), os.path.join(td, "c.json")
        np.save(qf, ds.queries[:nq_all])
        with open(cf, "w") as f:
            json.dump([[n, pred.to_json(p)] for n, p in classes], f)
        for prec, name in ((0, "fp32"), (1, "sq8")):
            res = {}
            for B in sizes:
                cmd = [sys.executable, "-m", "oracle.refgpu", "brute", "--index", path,
                       "--queries", qf, "--classes", cf, "--batch", str(B), "--topb", str(TOPK),
                       "--precision", str(prec), "--steps", str(reps[B]), "--mixed"]
                try:
                    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True,
                                       timeout=900)
                    if r.returncode != 0:
                        res[str(B)] = {"failed": (r.stderr or r.stdout).strip().splitlines()[-1:]}
                        continue
                    rl = json.loads(r.stdout.strip().splitlines()[-1])
                    res[str(B)] = {"qps_e2e": rl["qps_e2e"],
                                   "kernel_ms_per_call": rl["kernel_ms_per_call"]}
                except Exception as e:
                    res[str(B)] = {"failed": str(e)}
            out["reference_gpu"][name] = res
        for f in (path, qf, cf):
            os.unlink(f)
        os.rmdir(td)
    line = {"metric": "filtered top-10 QPS by batch size, 1M x 128 L2", "unit": "queries/s",
            "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
            "config": {"workload": "1M x 128 Gaussian-mixture rows, filters rotating per query "
                                   "through the six classes, top-10; calls of <= 1024 queries",
                       "rows": N_ROWS, "dim": DIM, "k": TOPK, "batches": sizes},
            "results": out}
    print(json.dumps(line), flush=True)


def shared_graph(vectors, rank, dist, cache):
    """Rank 0 builds the HNSW graph (or reloads this host's cached copy);
    after a barrier the other ranks load rank 0's copy instead of building
    their own."""
    from paves_b200.hnsw import build_or_load
    h = build_or_load(vectors, cache, 16, 200) if rank == 0 else None
    if dist:
        dist.barrier()
    if rank != 0:
        h = build_or_load(vectors, cache, 16, 200)
    return h


def parity_vs_reference(ans, exact, results):
    """Answers of the reference CPU BruteCursor (query c * BATCH + i of class
    c) against the plain exact FP32 path and the chosen path: queries whose
    ids, and whose FP32 distances, are identical."""
    out = {}
    for name, get in (("exact_fp32", lambda c: (exact[c][0], exact[c][1], exact[c][2])),
                      ("chosen", lambda c: (results[c][0], results[c][4], results[c][1]))):
        n = ids_eq = d_eq = 0
        for c in range(len(exact)):
            if name == "chosen" and c not in results:
                continue
            ids, dists, cnt = get(c)
            for i in range(BATCH):
                q = c * BATCH + i
                if q not in ans:
                    continue
                r_ids, r_d = ans[q]
                k = int(cnt[i])
                n += 1
                same = k == len(r_ids) and np.array_equal(ids[i, :k].astype(np.uint64), r_ids)
                ids_eq += int(same)
                d_eq += int(same and np.array_equal(dists[i, :k], r_d))
        out[name] = {"queries": n, "ids_equal": ids_eq, "dist_equal": d_eq}
    return out


def summarize_ref_gpu(rg, rg_ans, cpu_ans):
    """The reference GPU leg's numbers, with its answers checked against the
    reference CPU's (fp32: identical ids; sq8: recall@10)."""
    for name, per in rg_ans.items():
        if name not in rg or "failed" in rg[name]:
            continue
        n = eq = 0
        rec = []
        for c, (ids, cnt) in per.items():
            for i in range(ids.shape[0]):
                q = c * BATCH + i
                if q not in cpu_ans:
                    continue
                r_ids = cpu_ans[q][0]
                k = int(cnt[i])
                n += 1
                eq += int(k == len(r_ids) and np.array_equal(ids[i, :k].astype(np.uint64), r_ids))
                if len(r_ids):
                    rec.append(np.isin(r_ids, ids[i, :k]).mean())
        rg[name]["vs_reference_cpu"] = {"queries": n, "ids_equal": eq,
                                        "recall_at_10": round(float(np.mean(rec)), 4)
                                        if rec else None}
    return rg


def reduce_max(vals, dist, device):
    """Element-wise max over ranks (the job's time is its slowest rank's)."""
    if not dist:
        return list(vals)
    import torch
    t = torch.tensor(vals, device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the baseline legs (reference CPU, reference GPU, parity)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the reference GPU leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the graph points (1M x 128 at ef 32..256) and the uneven "
                         "micro-batch stream (10M x 96) reported beside the headline")
    ap.add_argument("--workload", default="headline",
                    choices=["headline", "stream", "graph", "batches"],
                    help="stream: uneven micro-batches over 10M x 96 FP8 (p50/p99 latency); "
                         "graph: filtered HNSW search at ef 32..256 beside the reference cursor; "
                         "batches: batch sizes 1..4096 beside the reference GPU kernels")
    ap.add_argument("--kernel-case", choices=sorted(KERNEL_CASES),
                    help="run one batch shape --steps times and exit (for profilers)")
    ap.add_argument("--tc-shape", default=None,
                    help="kernel cases: tensor-core shape epi,stages,grow,replicas,seed "
                         "(0 = auto; seed 2 = no seeding pass)")
    args = ap.parse_args()
    if args.workload == "stream":
        stream_bench(args)
        return
    if args.workload == "graph":
        graph_bench(args)
        return
    if args.workload == "batches":
        batches_bench(args)
        return
    if args.kernel_case:
        shape = None
        if args.tc_shape:
            shape = tuple(int(x) for x in args.tc_shape.split(","))
            shape = shape + (0,) * (5 - len(shape))
        kernel_case(args.kernel_case, max(1, args.steps), shape)
        return
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    ds, classes, preds_all = make_workload()
    nclass = len(classes)
    from paves_b200.router import Router, routed_batch
    cache = os.path.join(tempfile.gettempdir(), f"paves_bench_hnsw_{N_ROWS}x{DIM}.npz")
    t_build = time.perf_counter()
    hnsw = shared_graph(ds.vectors, rank, dist, cache)
    build_s = time.perf_counter() - t_build
    gi = GpuIndex(ds.vectors, ds.cols, l0=hnsw.l0, device=local,
                  precision=_lib.FV_GPU_PREC_BF16)
    if not os.path.exists(ROUTER_FILE):
        raise RuntimeError(f"{ROUTER_FILE} missing: train it with "
                           "python -m paves_b200.router_train --out " + ROUTER_FILE)
    z = np.load(ROUTER_FILE)
    router = Router(z["centroids"].astype(np.float32), device=local)
    router.set_params(z["params"], z["mean"], z["std"])
    L = _lib.lib()
    cls = []
    for c, (name, p) in enumerate(classes):
        q = np.ascontiguousarray(ds.queries[c * BATCH:(c + 1) * BATCH], np.float32)
        ent = hnsw.entries(q)
        bp = pred.concat([p] * BATCH, N_ROWS, entries=ent)
        cls.append((name, p, q, ent, bp))

    # plain path: exact FP32 scan of each class batch (prepared, resident):
    # on the tensor cores (f32 rows read as TF32, certified exact), and on
    # the CUDA cores alone (pv_exact_tc off)
    per_class = max(1, args.steps // nclass)

    def plain_leg():
        # (stage events: stage 1 is the scan kernel of each batch)
        bxs, ms_tot, on_tc, scan_tc_ms = [], 0.0, 0, []
        for name, p, q, ent, bp in cls:
            bx = prepared_batch(gi, q, bp, TOPK, _lib.PV_MODE_EXACT)
            batch_run(bx, 3)
            _, st = batch_run(bx, per_class, stages=True)
            ms_tot += sum(st)
            if L.pv_last_exact_tc(gi.handle):
                on_tc += 1
                if not L.pv_last_sparse(gi.handle):  # a pass over the whole index
                    scan_tc_ms.append(st[1] / per_class)
            bxs.append(bx)
        ans = [fetch(bx, BATCH, TOPK) for bx in bxs]
        for bx in bxs:
            L.pv_batch_free(bx)
        return BATCH * per_class * nclass / (ms_tot / 1e3), ans, on_tc, scan_tc_ms

    plain_qps, exact, plain_tc, tf32_ms = plain_leg()
    L.pv_exact_tc(gi.handle, 0)
    simt_qps, exact_simt, _, _ = plain_leg()
    L.pv_exact_tc(gi.handle, 1)
    simt_same = all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
                    for a, b in zip(exact, exact_simt))

    def routed(c):
        name, p, q, ent, bp = cls[c]
        return routed_batch(gi, router, q, None, TOPK, ent, topb=TOPK, bp=bp)

    for i in range(args.warmup):
        routed(i % nclass)

    def barrier():
        if dist:
            import torch
            t = torch.zeros(1, device=f"cuda:{local}")
            dist.all_reduce(t)
            torch.cuda.synchronize()

    barrier()
    clk = Clocks(local)
    dev_ms, launches, graph_steps, mixed_steps = 0.0, 0, 0, 0
    st_sum = np.zeros(3)
    results = {}
    cls_ms = {}
    t0 = time.perf_counter()
    for i in range(args.steps):
        c = i % nclass
        ids, dists, cnt, dec, ex, st = routed(c)
        dev_ms += float(st[0] + st[2])  # bitmaps, then the search (routing beside)
        cls_ms.setdefault(c, []).append(float(st[0] + st[2]))
        st_sum += st
        launches += int(L.pv_last_launches(gi.handle))
        graph_steps += int(ex == 1)
        mixed_steps += int(ex == 2)
        results[c] = (ids, cnt, dec, ex, dists)
    wall_s = time.perf_counter() - t0
    clocks = clk.stop()
    barrier()
    dev_ms, wall_s = reduce_max([dev_ms, wall_s], dist, f"cuda:{local}")
    ms_per_step = dev_ms / args.steps
    value = BATCH * args.steps * world / (dev_ms / 1e3)
    e2e_qps = BATCH * args.steps * world / wall_s
    recall = {}
    for c, (name, *_rest) in enumerate(cls):
        if c not in results:
            continue
        ids, cnt, dec, ex, _ = results[c]
        xi, _, xc, _ = exact[c]
        r = [np.isin(xi[i, :xc[i]], ids[i, :cnt[i]]).sum() / max(1, int(xc[i]))
             for i in range(BATCH)]
        recall[name] = {"recall_at_10": round(float(np.mean(r)), 4),
                        "ms": round(float(np.mean(cls_ms[c])), 4),
                        "path": {0: "bf16-scan", 1: "graph", 2: "mixed"}[int(ex)],
                        "graph_queries": int((dec > 0).sum())}

    # the scan path without the router (each class batch, prepared); the
    # roofline averages the tensor-core kernel over the classes that run it
    # (selective classes take the sparse route: an exact scan of their rows)
    st_tot, st_tc, n_tc, superset, per_cls = [0.0] * 4, [0.0] * 4, 0, 0, {}
    for name, p, q, ent, bp in cls:
        b = prepared_batch(gi, q, bp, TOPK, _lib.PV_MODE_LOW)
        batch_run(b, 3)
        _, st = batch_run(b, per_class, stages=True)
        sparse = bool(L.pv_last_sparse(gi.handle))
        st_tot = [x + y for x, y in zip(st_tot, st)]
        if not sparse:
            st_tc = [x + y for x, y in zip(st_tc, st)]
            n_tc += per_class
            superset = int(L.pv_last_superset(gi.handle))
        per_cls[name] = {"route": "sparse" if sparse else "tensor-core",
                         "ms": round(sum(st) / per_class, 4)}
        L.pv_batch_free(b)
    nrun = per_class * nclass
    scan_ms = st_tc[1] / max(1, n_tc)
    scan_only_qps = BATCH * nrun / (sum(st_tot) / 1e3)
    hbm, bf16, peak_kind = load_peaks()
    # tensor-core scan: bf16 rows (128 dims = 256 B) + f32 norm, once per batch
    alg_bytes = N_ROWS * (DIM * 2 + 4)
    achieved = alg_bytes / (scan_ms / 1e3) / 1e9

    # scan GB/s at batch 1 (the HBM-bound exact scan)
    bp1 = pred.concat([classes[5][1]], N_ROWS)
    b1 = prepared_batch(gi, ds.queries[:1], bp1, TOPK, _lib.PV_MODE_EXACT)
    batch_run(b1, 3)
    _, st1 = batch_run(b1, 20, stages=True)
    scan1_ms = st1[1] / 20
    scan_gbs_b1 = N_ROWS * DIM * 4 / (scan1_ms / 1e3) / 1e9
    L.pv_batch_free(b1)

    # bytes crossing PCIe per step of the chosen path (from the arrays passed)
    name, p, q, ent, bp = cls[0]
    h2d = q.nbytes + bp.qd.nbytes + bp.nodes.nbytes + bp.children.nbytes + bp.invals.nbytes
    d2h = BATCH * TOPK * 16 + BATCH * 4 + BATCH * 2

    cpu, parity, ref_gpu = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import refengine
            with tempfile.TemporaryDirectory(dir="/tmp") as td:
                path = os.path.join(td, "bench.idx")
                write_brute_index(ds, path)
                if refengine.available("cpu"):
                    qps, nrun_c, threads, ans = reference_cpu_leg(path, ds, preds_all, 1, 1,
                                                                  keep=True)
                    cpu = {"value": round(qps, 2), "unit": "queries/s", "cores": threads,
                           "kind": "reference",
                           "sample": f"{nrun_c} queries (the six class batches), one at a "
                                     "time (BruteCursor), after one warm-up pass"}
                    parity = parity_vs_reference(ans, exact, results)
                if not args.no_ref_gpu:
                    rg, rg_ans = reference_gpu_leg(path, ds, classes, args.steps)
                    ref_gpu = summarize_ref_gpu(rg, rg_ans, ans if cpu else {})
        except Exception as e:  # baselines are informative only
            cpu = {"value": None, "unit": "queries/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": f"failed: {e}"}

    extras = rank == 0 and world == 1 and not args.no_extras
    graph_pts, stream_res = None, None
    if extras:  # the graph search alone on this index's graph (64 queries per point)
        qg = np.ascontiguousarray(ds.queries[:BATCH], np.float32)
        graph_pts = graph_points(gi, qg, hnsw.entries(qg), min(args.steps, 10), 1)
    router.close()
    gi.close()
    if extras:
        try:
            stream_res = stream_results(100, 5)
        except Exception as e:  # informative; the headline stands
            stream_res = {"failed": str(e)}
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic",
            "config": {"workload": "1M x 128 Gaussian-mixture rows (integer-valued), six "
                                   "64-query batches, one per filter class (0.1%-95%), "
                                   "filtered top-10; learned router over the BF16 "
                                   "tensor-core scan + exact FP32 re-rank and the HNSW "
                                   "graph search",
                       "rows": N_ROWS, "dim": DIM, "batch": BATCH, "k": TOPK,
                       "rerank_candidates": superset, "hnsw": "M=16 efC=200",
                       "l2_flush": "inputs larger than L2 (256 MB bf16 rows, 512 MB f32 "
                                   "rows vs 126 MB)"},
            "recall_per_class": recall,
            "recall_at_10_min": round(min(v["recall_at_10"] for v in recall.values()), 4),
            "graph_batches": graph_steps,
            "mixed_batches": mixed_steps,
            "routed_stage_ms": {"bitmaps": round(st_sum[0] / args.steps, 4),
                                "routing_after_bitmaps": round(st_sum[1] / args.steps, 4),
                                "search": round(st_sum[2] / args.steps, 4)},
            "plain_gpu": {"value": round(plain_qps, 1), "unit": "queries/s",
                          "path": "exact FP32 results: f32 rows read as TF32 on the tensor "
                                  "cores, certified exact (the sparse route for selective "
                                  "filters)",
                          "tensor_core_batches": f"{plain_tc} of {nclass}",
                          "cuda_cores_only": round(simt_qps, 1),
                          "same_answers_as_cuda_cores": simt_same},
            # the exact path's dominant kernel: f32 rows (512 B) + f32 norm per row
            "roofline_exact": None if not tf32_ms else {
                "bound": "hbm", "kernel": "scan_tc_kernel (TF32)", "unit": "GB/s",
                "achieved": round(N_ROWS * (DIM * 4 + 4) / (statistics.mean(tf32_ms) / 1e3) / 1e9, 1),
                "peak": hbm, "peak_kind": peak_kind,
                "frac": round(N_ROWS * (DIM * 4 + 4) / (statistics.mean(tf32_ms) / 1e3) / 1e9 / hbm, 4),
                "kernel_ms": round(statistics.mean(tf32_ms), 4),
                "alg_bytes_per_launch": N_ROWS * (DIM * 4 + 4),
                "traffic": load_traffic("scan_tc_kernel_tf32"),
                "traffic_source": "ncu capture of the same kernel (profiles/traffic.json)"},
            "scan_only": {"value": round(scan_only_qps, 1), "unit": "queries/s",
                          "path": "bf16 scan + re-rank (sparse route for selective "
                                  "filters), no router", "classes": per_cls},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(achieved / hbm, 4),
                         "traffic": load_traffic("scan_tc_kernel"),
                         "traffic_source": "ncu capture of the same kernel and workload "
                                           "(profiles/traffic.json), not this run",
                         "kernel": "scan_tc_kernel", "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg_bytes, "kernel_ms": round(scan_ms, 4)},
            "scan_gbs_batch1": round(scan_gbs_b1, 1),
            "stage_ms": {"bitmap+prep+seed": round(st_tc[0] / max(1, n_tc), 4),
                         "scan": round(scan_ms, 4),
                         "merge+rerank": round(st_tc[2] / max(1, n_tc), 4)},
            "hnsw_build_s": round(build_s, 1),
            "clocks": clocks,
            "e2e": {"value": round(e2e_qps, 1), "unit": "queries/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "cpu_baseline": cpu,
            "parity_vs_reference_cpu": parity,
            "reference_gpu": ref_gpu,
            "graph_search_points": graph_pts,
            "uneven_microbatches": None if stream_res is None else {
                "config": STREAM_CONFIG, "unit": "queries/s", "dtype": "fp8-e4m3",
                **stream_res},
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
