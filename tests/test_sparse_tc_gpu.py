"""The sparse route on the tensor cores: a batch whose queries share one
selective filter (bounded on the host at 16384+ matching rows) compacts the
matching rows and scans only them on the tensor cores (BF16 / FP8 rows, or
the f32 rows read as TF32 in the exact mode).

Bars: integer rows give the oracle's exact filtered top-k (ids, FP32
distances, counts, truncation flags) on BF16 and FP32 uploads; FP8 keeps
recall >= 0.99 with exact re-ranked distances; non-integer rows on an FP32
upload agree with the FP64 oracle to 1e-5 rank by rank."""
import numpy as np
import pytest

from oracle import cpu
from paves_b200 import (FV_GPU_PREC_BF16, FV_GPU_PREC_FP8, GpuIndex, _lib, datagen, pred)

pytestmark = pytest.mark.gpu
N, D = 1_000_003, 128
P, Cc = datagen.COL_PRICE, datagen.COL_CATEGORY

FILTERS = {
    # ~2 % of rows (price is uniform in [0, 1000)): ~20,000 rows
    "price<20": pred.Cmp(P, "<", 20.0),
    # ~1.2 %, two columns (bounded by the price term: ~40,000 rows)
    "price<40&cat3-5": pred.And(pred.Cmp(P, "<", 40.0), pred.In(Cc, [3.0, 4.0, 5.0])),
    # ~5 %: ~50,000 rows, still under the route's limit (rows / 16)
    "price<50": pred.Cmp(P, "<", 50.0),
    # ~0.3 %: below the tensor-core threshold, the CUDA-core sparse route
    "price<3": pred.Cmp(P, "<", 3.0),
}


@pytest.fixture(scope="module")
def ds():
    return datagen.make_dataset(N, D, nq=64)


def _exact(ds, gi, q, p, topb):
    bp = pred.concat([p] * len(q), N)
    ids, dists, cnt, trunc = gi.brute_batch_raw(q, bp, topb)
    assert _lib.lib().pv_last_sparse(gi.handle) == 1
    o_ids, _, o_d32, o_cnt, o_pass = cpu.exact_topk(ds.vectors, ds.cols, q, bp, topb)
    for i in range(len(q)):
        n = int(o_cnt[i])
        assert cnt[i] == n, i
        assert np.array_equal(ids[i, :n], o_ids[i, :n].astype(np.uint64)), i
        assert np.array_equal(dists[i, :n], o_d32[i, :n]), i
        assert trunc[i] == (o_pass[i] > topb), i


@pytest.fixture(scope="module")
def bf16(ds):
    gi = GpuIndex(ds.vectors, ds.cols, precision=FV_GPU_PREC_BF16)
    yield gi
    gi.close()


@pytest.fixture(scope="module")
def fp32(ds):
    gi = GpuIndex(ds.vectors, ds.cols)
    yield gi
    gi.close()


@pytest.mark.parametrize("name", list(FILTERS))
@pytest.mark.parametrize("topb", [10, 100])
def test_bf16_sparse_matches_oracle(ds, bf16, name, topb):
    _exact(ds, bf16, ds.queries, FILTERS[name], topb)


@pytest.mark.parametrize("name", list(FILTERS))
def test_fp32_exact_sparse_matches_oracle(ds, fp32, name):
    _exact(ds, fp32, ds.queries[:32], FILTERS[name], 10)
    if name != "price<3":
        assert _lib.lib().pv_last_exact_tc(fp32.handle) == 1


def test_fp8_sparse_recall(ds):
    gi = GpuIndex(ds.vectors, ds.cols, precision=FV_GPU_PREC_FP8)
    p = FILTERS["price<20"]
    bp = pred.concat([p] * 64, N)
    ids, dists, cnt, _ = gi.brute_batch_raw(ds.queries, bp, 10)
    assert _lib.lib().pv_last_sparse(gi.handle) == 1
    o_ids, _, _, o_cnt, _ = cpu.exact_topk(ds.vectors, ds.cols, ds.queries, bp, 10)
    hit = tot = 0
    for i in range(64):
        c = int(cnt[i])
        assert c == int(o_cnt[i])
        hit += np.isin(o_ids[i, :c], ids[i, :c]).sum()
        tot += c
        rows = ids[i, :c].astype(np.int64)
        exact = np.sum((ds.vectors[rows] - ds.queries[i]) ** 2, 1, dtype=np.float32)
        assert np.array_equal(dists[i, :c], exact)
    assert hit / tot >= 0.99
    gi.close()


def test_non_integer_rows_exact_mode(ds):
    rng = np.random.default_rng(7)
    vecs = (ds.vectors + rng.standard_normal(ds.vectors.shape) * 0.37).astype(np.float32)
    qs = (ds.queries[:32] + rng.standard_normal((32, D)) * 0.37).astype(np.float32)
    gi = GpuIndex(vecs, ds.cols)
    p = FILTERS["price<40&cat3-5"]
    bp = pred.concat([p] * 32, N)
    ids, dists, cnt, _ = gi.brute_batch_raw(qs, bp, 10)
    assert _lib.lib().pv_last_sparse(gi.handle) == 1
    o_ids, o_d64, _, o_cnt, _ = cpu.exact_topk(vecs, ds.cols, qs, bp, 10)
    for i in range(32):
        k = int(o_cnt[i])
        assert cnt[i] == k
        np.testing.assert_allclose(dists[i, :k], o_d64[i, :k], rtol=1e-5)
    gi.close()
