"""Reduced-precision scans on the tensor cores (BF16 / FP8-E4M3 distances,
exact FP32 re-rank of a 4k-candidate superset) through the C ABI.

Bars: on integer-valued rows BF16 distances are exact, so the BF16 path
must return exactly the reference's top-k (ids and distances); returned
distances are always the exact FP32 ones (re-ranked); FP8 keeps
recall@10 >= 0.95 per query batch; non-integer rows keep recall >= 0.99
with BF16."""
import numpy as np
import pytest

from oracle import cpu
from paves_b200 import FV_GPU_PREC_BF16, FV_GPU_PREC_FP8, FV_GPU_PREC_SQ8, GpuIndex, datagen, pred

pytestmark = pytest.mark.gpu


def recall(ids, o_ids, o_cnt, k):
    tot = hit = 0
    for q in range(ids.shape[0]):
        t = set(o_ids[q, :min(k, o_cnt[q])].tolist())
        hit += len(t & set(ids[q, :k].tolist()))
        tot += len(t)
    return hit / max(tot, 1)


@pytest.fixture(scope="module")
def bf16_golden(brute_golden):
    g = brute_golden
    return GpuIndex(g["vectors"], g["cols"], precision=FV_GPU_PREC_BF16)


def test_bf16_integer_rows_match_reference(bf16_golden, brute_golden):
    g = brute_golden
    nq = g["queries"].shape[0]
    assert bf16_golden.precision == FV_GPU_PREC_BF16
    for pi, p in enumerate(g["preds"]):
        ids, dists, cnt, trunc = bf16_golden.brute_batch(g["queries"], [p] * nq, 10)
        for q in range(nq):
            n = int((g["ids10"][pi, q] >= 0).sum())
            assert cnt[q] == n, (pi, q)
            assert np.array_equal(ids[q, :n].astype(np.int64), g["ids10"][pi, q, :n]), (pi, q)
            assert np.array_equal(dists[q, :n], g["d10"][pi, q, :n]), (pi, q)


@pytest.mark.parametrize("nq,topb", [(1, 10), (64, 10), (300, 16), (129, 1), (40, 5)])
def test_bf16_large_vs_oracle(nq, topb):
    ds = datagen.make_dataset(150_001, 128, nq=nq)
    gi = GpuIndex(ds.vectors, ds.cols, precision=FV_GPU_PREC_BF16)
    six = list(datagen.six_predicates().values()) + [None]
    preds = [six[q % len(six)] for q in range(nq)]
    bp = pred.concat(preds, len(ds.vectors))
    ids, dists, cnt, trunc = gi.brute_batch_raw(ds.queries, bp, topb)
    o_ids, _, o_d32, o_cnt, o_pass = cpu.exact_topk(ds.vectors, ds.cols, ds.queries, bp, topb)
    for q in range(nq):
        n = int(o_cnt[q])
        assert cnt[q] == n
        assert np.array_equal(ids[q, :n], o_ids[q, :n].astype(np.uint64)), q
        assert np.array_equal(dists[q, :n], o_d32[q, :n]), q
        assert trunc[q] == (o_pass[q] > topb)
    gi.close()


@pytest.mark.parametrize("n,d,prec", [(20000, 96, FV_GPU_PREC_FP8), (20000, 128, FV_GPU_PREC_FP8),
                                      (9000, 100, FV_GPU_PREC_BF16), (9000, 256, FV_GPU_PREC_BF16),
                                      (9000, 256, FV_GPU_PREC_FP8), (5000, 64, FV_GPU_PREC_SQ8)])
def test_precisions_recall_and_exact_distances(n, d, prec):
    ds = datagen.make_dataset(n, d, nq=64, ncomp=64)
    gi = GpuIndex(ds.vectors, ds.cols, precision=prec)
    preds = [None, datagen.six_predicates()["sel30%"], datagen.six_predicates()["sel70%"]] * 22
    bp = pred.concat(preds[:64], n)
    ids, dists, cnt, _ = gi.brute_batch_raw(ds.queries, bp, 10)
    o_ids, _, _, o_cnt, _ = cpu.exact_topk(ds.vectors, ds.cols, ds.queries, bp, 10)
    r = recall(ids.astype(np.int64), o_ids.astype(np.int64), o_cnt, 10)
    assert r >= (0.95 if prec == FV_GPU_PREC_FP8 else 0.999), r
    for q in range(64):
        c = int(cnt[q])
        rows = ids[q, :c].astype(np.int64)
        exact = np.sum((ds.vectors[rows] - ds.queries[q]) ** 2, 1, dtype=np.float32)
        assert np.array_equal(dists[q, :c], exact)
        assert np.all(np.diff(dists[q, :c]) >= 0)
    gi.close()


def test_bf16_non_integer_rows_recall():
    rng = np.random.default_rng(3)
    vecs = rng.standard_normal((30000, 128)).astype(np.float32)
    qs = rng.standard_normal((64, 128)).astype(np.float32)
    cols = rng.uniform(0, 1000, (2, 30000))
    gi = GpuIndex(vecs, cols, precision=FV_GPU_PREC_BF16)
    bp = pred.concat([None, pred.Cmp(1, "<", 300.0)] * 32, 30000)
    ids, dists, cnt, _ = gi.brute_batch_raw(qs, bp, 10)
    o_ids, _, _, o_cnt, _ = cpu.exact_topk(vecs, cols, qs, bp, 10)
    assert recall(ids.astype(np.int64), o_ids.astype(np.int64), o_cnt, 10) >= 0.99
    gi.close()


def test_large_topb_falls_back_to_exact(bf16_golden, brute_golden):
    g = brute_golden
    nq = g["queries"].shape[0]
    ids, dists, cnt, _ = bf16_golden.brute_batch(g["queries"], [None] * nq, 100)
    for q in range(nq):
        assert np.array_equal(ids[q].astype(np.int64), g["ids100"][0, q])


@pytest.mark.parametrize("clustered", [False, True])
def test_fp8_large_k_superset_certified_or_rerun(clustered):
    """k = 100 on FP8 keeps a 400-candidate superset from per-CTA lists of
    64; queries whose superset cannot be certified are re-run exactly. With
    rows stored cluster by cluster, a query's nearest rows crowd a few lists,
    so most queries take the exact re-run."""
    from paves_b200 import _lib
    ds = datagen.make_dataset(20000, 96, nq=32, ncomp=64)
    vecs, cols = ds.vectors, ds.cols
    if clustered:
        order = np.argsort(((vecs[:, None, :8] - ds.centers[None, :, :8]) ** 2).sum(2).argmin(1),
                           kind="stable")
        vecs, cols = np.ascontiguousarray(vecs[order]), np.ascontiguousarray(cols[:, order])
    gi = GpuIndex(vecs, cols, precision=FV_GPU_PREC_FP8)
    # one epilogue group, no query replicas: each list then sees all 128 rows
    # of its CTA's tiles (512 rows), more than its 64 keys (with replicas a
    # list can see as few rows as it holds, and never drop one)
    assert _lib.lib().pv_tc_shape(gi.handle, 1, 0, 0, 1, 0) == 0
    preds = [None, datagen.six_predicates()["sel70%"]] * 16
    bp = pred.concat(preds, 20000)
    ids, dists, cnt, _ = gi.brute_batch_raw(ds.queries, bp, 100)
    unc = _lib.lib().pv_last_uncertain(gi.handle)
    assert _lib.lib().pv_last_superset(gi.handle) == 400
    o_ids, _, _, o_cnt, _ = cpu.exact_topk(vecs, cols, ds.queries, bp, 100)
    r = recall(ids.astype(np.int64), o_ids.astype(np.int64), o_cnt, 100)
    assert r >= 0.99, (r, unc)
    if clustered:
        assert unc > 0
    for q in range(32):
        c = int(cnt[q])
        assert c == int(o_cnt[q])
        rows = ids[q, :c].astype(np.int64)
        exact = np.sum((vecs[rows] - ds.queries[q]) ** 2, 1, dtype=np.float32)
        assert np.array_equal(dists[q, :c], exact)
        assert np.all(np.diff(dists[q, :c]) >= 0)
    gi.close()


@pytest.mark.parametrize("epi,rep,nq", [(1, 4, 1), (1, 4, 24), (2, 2, 24), (1, 2, 64),
                                        (2, 2, 64), (2, 1, 64), (1, 1, 40), (2, 4, 16),
                                        (3, 2, 64), (3, 1, 100), (3, 4, 7)])
def test_tc_epilogue_shapes_match_oracle(epi, rep, nq):
    """Every epilogue shape (warp groups x query replicas down the tile)
    returns exactly the oracle's top-k on integer rows: replicas split each
    tile's rows, so a lost or doubly counted row would show here."""
    from paves_b200 import _lib
    L = _lib.lib()
    ds = datagen.make_dataset(90_001, 128, nq=nq)
    gi = GpuIndex(ds.vectors, ds.cols, precision=FV_GPU_PREC_BF16)
    assert L.pv_tc_shape(gi.handle, epi, 0, 0, rep, 2 if rep == 2 else 0) == 0
    six = list(datagen.six_predicates().values()) + [None]
    preds = [six[(q + 3) % len(six)] for q in range(nq)]
    bp = pred.concat(preds, len(ds.vectors))
    for topb in (1, 10):
        ids, dists, cnt, trunc = gi.brute_batch_raw(ds.queries, bp, topb)
        assert L.pv_last_sparse(gi.handle) == 0 and L.pv_last_superset(gi.handle) > 0
        o_ids, _, o_d32, o_cnt, o_pass = cpu.exact_topk(ds.vectors, ds.cols, ds.queries, bp, topb)
        for q in range(nq):
            n = int(o_cnt[q])
            assert cnt[q] == n, (q, topb)
            assert np.array_equal(ids[q, :n], o_ids[q, :n].astype(np.uint64)), (q, topb)
            assert np.array_equal(dists[q, :n], o_d32[q, :n]), (q, topb)
            assert trunc[q] == (o_pass[q] > topb)
    assert L.pv_tc_shape(gi.handle, 0, 0, 0, 3, 0) == -1
    gi.close()


def test_fresh_fp8_indexes_convert_every_row():
    """Uploads order their copies, fills and the FP8 conversion on one
    stream: a fill left on the default stream once raced the conversion
    and zeroed row scales of about one FP8 index in a hundred (rows then
    looked far from every query). Many fresh small indexes, one batch
    each, all at the recall bar."""
    n, d = 5000, 96
    ds = datagen.make_dataset(n, d, nq=32, ncomp=64)
    bp = pred.concat([None, datagen.six_predicates()["sel70%"]] * 16, n)
    o_ids, _, _, o_cnt, _ = cpu.exact_topk(ds.vectors, ds.cols, ds.queries, bp, 10)
    for i in range(200):
        gi = GpuIndex(ds.vectors, ds.cols, precision=FV_GPU_PREC_FP8)
        ids, _, _, _ = gi.brute_batch_raw(ds.queries, bp, 10)
        gi.close()
        r = recall(ids.astype(np.int64), o_ids.astype(np.int64), o_cnt, 10)
        assert r >= 0.95, (i, r)
