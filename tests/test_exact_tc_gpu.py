"""The exact mode on the tensor cores: batches of 16+ queries read the f32
rows as TF32 (tcgen05 kind::tf32), re-rank a superset in FP32 and certify
each query's answer by an error bound of the scan distances; queries the
bound cannot separate are re-run on the CUDA-core scan.

Bars: on integer rows (the reference's benchmark data) the answer is the
oracle's exactly, ids and distances, as the CUDA-core scan's is; on
non-integer rows the distances agree with the oracle's FP64 ones to the
FP32 tolerance of the CUDA-core scan's own test, rank by rank; rows the
bound cannot separate (near-equal distances) fall back and return exactly
what the CUDA-core scan returns."""
import numpy as np
import pytest

from oracle import cpu
from paves_b200 import GpuIndex, _lib, datagen, pred

pytestmark = pytest.mark.gpu


def _exact_tc(gi, on):
    assert _lib.lib().pv_exact_tc(gi.handle, 1 if on else 0) == 0


def _took_tc(gi):
    return _lib.lib().pv_last_exact_tc(gi.handle) == 1


def _uncertain(gi):
    return _lib.lib().pv_last_uncertain(gi.handle)


@pytest.fixture(scope="module")
def ints():
    ds = datagen.make_dataset(150_001, 128, nq=300)
    gi = GpuIndex(ds.vectors, ds.cols)  # FP32 upload: the drop-in's exact mode
    yield ds, gi
    gi.close()


@pytest.mark.parametrize("nq,topb", [(16, 10), (64, 10), (64, 100), (200, 1), (300, 64)])
def test_integer_rows_match_oracle_exactly(ints, nq, topb):
    ds, gi = ints
    six = list(datagen.six_predicates().values()) + [None]
    preds = [six[q % len(six)] for q in range(nq)]
    bp = pred.concat(preds, len(ds.vectors))
    q = ds.queries[:nq]
    ids, dists, cnt, trunc = gi.brute_batch_raw(q, bp, topb)
    assert _took_tc(gi)
    assert _uncertain(gi) == 0  # integer rows: the scan distances are exact
    o_ids, _, o_d32, o_cnt, o_pass = cpu.exact_topk(ds.vectors, ds.cols, q, bp, topb)
    for i in range(nq):
        n = int(o_cnt[i])
        assert cnt[i] == n, i
        assert np.array_equal(ids[i, :n], o_ids[i, :n].astype(np.uint64)), i
        assert np.array_equal(dists[i, :n], o_d32[i, :n]), i
        assert trunc[i] == (o_pass[i] > topb), i


def test_small_batches_stay_on_the_cuda_cores(ints):
    ds, gi = ints
    ids, dists, cnt, _ = gi.brute_batch(ds.queries[:15], [None] * 15, 10)
    assert not _took_tc(gi)
    _exact_tc(gi, False)
    try:
        i2, d2, c2, _ = gi.brute_batch(ds.queries[:64], [None] * 64, 10)
        assert not _took_tc(gi)
    finally:
        _exact_tc(gi, True)
    i3, d3, c3, _ = gi.brute_batch(ds.queries[:64], [None] * 64, 10)
    assert _took_tc(gi)
    assert np.array_equal(i2, i3) and np.array_equal(d2, d3) and np.array_equal(c2, c3)


@pytest.mark.parametrize("n,d", [(20_011, 100), (9_000, 36), (66_000, 128)])
def test_ragged_dims_and_counts(n, d):
    rng = np.random.default_rng(n + d)
    vecs = rng.integers(0, 200, (n, d)).astype(np.float32)
    cols = np.stack([rng.integers(0, 10, n).astype(np.float64), rng.uniform(0, 1000, n)])
    qs = rng.integers(0, 200, (40, d)).astype(np.float32)
    gi = GpuIndex(vecs, cols)
    preds = [None, pred.Cmp(1, "<", 300.0), pred.In(0, [1.0, 2.0, 7.0])] * 14
    bp = pred.concat(preds[:40], n)
    ids, dists, cnt, _ = gi.brute_batch_raw(qs, bp, 10)
    assert _took_tc(gi)
    o_ids, _, o_d32, o_cnt, _ = cpu.exact_topk(vecs, cols, qs, bp, 10)
    for i in range(40):
        k = int(o_cnt[i])
        assert cnt[i] == k
        assert np.array_equal(ids[i, :k], o_ids[i, :k].astype(np.uint64)), i
        assert np.array_equal(dists[i, :k], o_d32[i, :k]), i
    gi.close()


@pytest.mark.parametrize("topb", [1, 10, 100])
def test_non_integer_rows_within_tolerance(topb):
    ds = datagen.make_dataset(100_000, 96, nq=64)
    rng = np.random.default_rng(5)
    vecs = (ds.vectors + rng.standard_normal(ds.vectors.shape) * 0.37).astype(np.float32)
    qs = (ds.queries + rng.standard_normal(ds.queries.shape) * 0.37).astype(np.float32)
    gi = GpuIndex(vecs, ds.cols)
    six = list(datagen.six_predicates().values())
    preds = [six[q % len(six)] for q in range(64)]
    bp = pred.concat(preds, len(vecs))
    ids, dists, cnt, _ = gi.brute_batch_raw(qs, bp, topb)
    assert _took_tc(gi)
    unc = _uncertain(gi)
    assert unc <= 8, unc  # the bound separates almost every query
    o_ids, o_d64, _, o_cnt, _ = cpu.exact_topk(vecs, ds.cols, qs, bp, topb)
    hit = tot = 0
    for i in range(64):
        k = int(o_cnt[i])
        assert cnt[i] == k
        np.testing.assert_allclose(dists[i, :k], o_d64[i, :k], rtol=1e-5)
        rows = ids[i, :k].astype(np.int64)
        true = np.sum((vecs[rows].astype(np.float64) - qs[i]) ** 2, 1)
        np.testing.assert_allclose(dists[i, :k], true, rtol=1e-5)
        hit += np.isin(o_ids[i, :k], ids[i, :k]).sum()
        tot += k
    assert hit / tot >= 0.999
    gi.close()


def test_unseparable_rows_fall_back_to_the_cuda_core_scan():
    # rows scattered 1e-4 around one point: every distance lies within the
    # scan's error bound of every other, so no query can be certified
    rng = np.random.default_rng(11)
    n, d = 40_000, 64
    center = rng.uniform(50, 60, d).astype(np.float32)
    vecs = (center + rng.standard_normal((n, d)) * 1e-4).astype(np.float32)
    qs = (center + rng.uniform(5, 6, (32, d))).astype(np.float32)
    gi = GpuIndex(vecs, None)
    ids, dists, cnt, _ = gi.brute_batch(qs, [None] * 32, 10)
    assert _took_tc(gi)
    assert _uncertain(gi) == 32
    _exact_tc(gi, False)
    i2, d2, c2, _ = gi.brute_batch(qs, [None] * 32, 10)
    assert np.array_equal(ids, i2) and np.array_equal(dists, d2) and np.array_equal(cnt, c2)
    gi.close()
