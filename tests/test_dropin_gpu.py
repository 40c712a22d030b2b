"""The drop-in proof, executed: the reference engine compiled from its own
unmodified sources with its GPU backend switched on (engine.cpp -DFV_GPU)
and linked against libpaves_gpu.so in place of gpu_engine.cu
(oracle/_ref/libpaves_ref_dropin.so). Through the engine's own batch calls
(fv_index_gpu_ensure, engine.cpp:1515-1535; fv_gpu_exec_brute_batch /
fv_gpu_exec_graph_batch, engine.cpp:1290-1339, which build GpuConcat
arrays and call this library's gpu_engine.h entry points) the results
must be the oracle's exact filtered top-k (brute, FP32 and BF16 uploads),
and the graph search must return what this library's own graph call
returns for the same graph, entries and ef."""
import os
import tempfile

import numpy as np
import pytest

from oracle import cpu, refengine
from paves_b200 import GpuIndex, datagen, pred
from paves_b200.hnsw import Hnsw

pytestmark = pytest.mark.gpu

N, D, NQ = 30_011, 128, 48


@pytest.fixture(scope="module")
def setup():
    if not refengine.available("dropin"):
        pytest.skip("oracle/_ref/libpaves_ref_dropin.so not built")
    ds = datagen.make_dataset(N, D, nq=NQ)
    h = Hnsw(ds.vectors, 16, 100)
    td = tempfile.mkdtemp(dir="/tmp")
    path = os.path.join(td, "dropin.idx")
    h.write(path, ds.cols)
    classes = list(datagen.six_predicates().values()) + [datagen.config1_predicate(), None]
    yield ds, h, path, classes
    os.unlink(path)
    os.rmdir(td)


@pytest.mark.parametrize("precision", [0, 2])  # FP32, BF16 (+ exact re-rank)
def test_engine_brute_batch_runs_our_kernels(setup, precision):
    ds, h, path, classes = setup
    R = refengine.RefIndex(path, kind="dropin")
    R.gpu_precision(precision)
    handles = [R.compile(p) for p in classes]
    ser = [R.serialize(x) for x in handles]
    preds = [classes[q % len(classes)] for q in range(NQ)]
    bps = [ser[q % len(classes)][0] for q in range(NQ)]
    for topb in (10, 64):
        ids, dists, cnt, trunc = R.gpu_brute_batch(ds.queries, bps, topb)
        bp = pred.concat(preds, N)
        o_ids, _, o_d32, o_cnt, o_pass = cpu.exact_topk(ds.vectors, ds.cols, ds.queries, bp, topb)
        assert np.array_equal(cnt, o_cnt)
        for q in range(NQ):
            n = int(o_cnt[q])
            assert np.array_equal(ids[q, :n], o_ids[q, :n].astype(np.uint64)), (topb, q)
            assert np.array_equal(dists[q, :n], o_d32[q, :n]), (topb, q)
            assert trunc[q] == (1 if o_pass[q] > topb else 0), (topb, q)
    for x in handles:
        R.free_pred(x)
    R.close()


def test_engine_graph_batch_runs_our_kernels(setup):
    ds, h, path, classes = setup
    R = refengine.RefIndex(path, kind="dropin")
    R.gpu_precision(0)
    entries = np.array([R.graph_entry(q) for q in ds.queries], np.uint32)
    # the engine's upper-level descent and this library's agree
    assert np.array_equal(entries, h.entries(ds.queries))
    gi = GpuIndex(ds.vectors, ds.cols, l0=h.l0)
    for p in (datagen.graph_predicates()["sel10%"], None):
        hp = R.compile(p)
        ser = R.serialize(hp)  # keeps the buffers the struct points into
        bp = ser[0]
        for ef in (32, 128):
            ids, dists, cnt, exh = R.gpu_graph_batch(ds.queries, entries, [bp] * NQ, ef,
                                                     max(200000, 400 * ef))
            g_ids, g_d, g_cnt, g_exh = gi.graph_batch(ds.queries, entries, [p] * NQ, ef)
            assert np.array_equal(cnt, g_cnt)
            assert np.array_equal(exh, g_exh)
            for q in range(NQ):
                c = int(cnt[q])
                assert np.array_equal(ids[q, :c], g_ids[q, :c]), (ef, q)
                assert np.array_equal(dists[q, :c], g_d[q, :c]), (ef, q)
        R.free_pred(hp)
    gi.close()
    R.close()
