"""Parity of the exact FP32 filtered scan (fv_gpu_brute_batch through the
C ABI) with the reference's golden outputs and with the oracle.

Bar: ids bit-identical and distances bit-identical (FP32 distances are
exact on integer-valued rows); for non-integer rows distances within
1e-5 relative of the FP64 oracle and ids identical except where FP32
rounding reorders near-ties (checked by distance)."""
import numpy as np
import pytest

from oracle import cpu
from paves_b200 import GpuError, GpuIndex, datagen, pred

pytestmark = pytest.mark.gpu


def check_exact(ids, dists, cnt, trunc, o_ids, o_d32, o_cnt, o_pass, topb):
    nq = ids.shape[0]
    for q in range(nq):
        n = int(o_cnt[q])
        assert cnt[q] == n, (q, cnt[q], n)
        assert np.array_equal(ids[q, :n], o_ids[q, :n].astype(np.uint64)), q
        assert np.array_equal(dists[q, :n], o_d32[q, :n]), q
        assert trunc[q] == (1 if o_pass[q] > topb else 0), q


@pytest.fixture(scope="module")
def golden_index(brute_golden):
    g = brute_golden
    return GpuIndex(g["vectors"], g["cols"])


@pytest.mark.parametrize("k", [10, 100])
def test_golden_reference_parity(golden_index, brute_golden, k):
    g = brute_golden
    nq = g["queries"].shape[0]
    gid, gd = (g["ids10"], g["d10"]) if k == 10 else (g["ids100"], g["d100"])
    for pi, p in enumerate(g["preds"]):
        ids, dists, cnt, trunc = golden_index.brute_batch(g["queries"], [p] * nq, k)
        for q in range(nq):
            n = int((gid[pi, q] >= 0).sum())
            assert cnt[q] == n, (pi, q)
            assert np.array_equal(ids[q, :n].astype(np.int64), gid[pi, q, :n]), (pi, q)
            assert np.array_equal(dists[q, :n], gd[pi, q, :n]), (pi, q)


def test_mixed_predicates_one_batch(golden_index, brute_golden):
    g = brute_golden
    nq = g["queries"].shape[0]
    preds = [g["preds"][q % len(g["preds"])] for q in range(nq)]
    bp = pred.concat(preds, g["vectors"].shape[0])
    for topb in (1, 10, 64, 257):
        ids, dists, cnt, trunc = golden_index.brute_batch_raw(g["queries"], bp, topb)
        o = cpu.exact_topk(g["vectors"], g["cols"], g["queries"], bp, topb)
        check_exact(ids, dists, cnt, trunc, o[0], o[2], o[3], o[4], topb)


@pytest.fixture(scope="module")
def big():
    ds = datagen.make_dataset(200_003, 128, nq=300)
    return ds, GpuIndex(ds.vectors, ds.cols)


@pytest.mark.parametrize("nq,topb", [(1, 10), (7, 64), (64, 10), (300, 100), (16, 1)])
def test_large_scan_vs_oracle(big, nq, topb):
    ds, gi = big
    six = list(datagen.six_predicates().values()) + [None, datagen.config1_predicate()]
    preds = [six[q % len(six)] for q in range(nq)]
    bp = pred.concat(preds, ds.vectors.shape[0])
    q = ds.queries[:nq]
    ids, dists, cnt, trunc = gi.brute_batch_raw(q, bp, topb)
    o = cpu.exact_topk(ds.vectors, ds.cols, q, bp, topb)
    check_exact(ids, dists, cnt, trunc, o[0], o[2], o[3], o[4], topb)


def test_max_topb(big):
    ds, gi = big
    preds = [None, datagen.six_predicates()["sel10%"], datagen.six_predicates()["sel0.1%"]]
    bp = pred.concat(preds, ds.vectors.shape[0])
    ids, dists, cnt, trunc = gi.brute_batch_raw(ds.queries[:3], bp, 4096)
    o = cpu.exact_topk(ds.vectors, ds.cols, ds.queries[:3], bp, 4096)
    check_exact(ids, dists, cnt, trunc, o[0], o[2], o[3], o[4], 4096)


@pytest.mark.parametrize("n,d", [(1007, 96), (777, 100), (5000, 256), (3000, 512), (5, 16),
                                 (31, 128), (33, 3)])
def test_shapes_vs_oracle(n, d):
    rng = np.random.default_rng(n * 7 + d)
    vecs = rng.integers(0, 256, (n, d)).astype(np.float32)
    cols = np.stack([rng.integers(0, 10, n).astype(np.float64), rng.uniform(0, 1000, n)])
    qs = rng.integers(0, 256, (9, d)).astype(np.float32)
    gi = GpuIndex(vecs, cols)
    preds = [None, pred.Cmp(1, "<", 300.0), pred.In(0, [1, 2]), pred.Cmp(1, "<", -5.0)] * 3
    bp = pred.concat(preds[:9], n)
    for topb in (1, 10, 50):
        ids, dists, cnt, trunc = gi.brute_batch_raw(qs, bp, topb)
        o = cpu.exact_topk(vecs, cols, qs, bp, topb)
        check_exact(ids, dists, cnt, trunc, o[0], o[2], o[3], o[4], topb)
    gi.close()


def test_ties_break_by_id():
    rng = np.random.default_rng(5)
    base = rng.integers(0, 4, (50, 32)).astype(np.float32)
    vecs = np.repeat(base, 200, axis=0)  # 10k rows, each distinct row x200
    rng.shuffle(vecs)
    cols = np.zeros((1, len(vecs)))
    qs = base[:8].copy()
    gi = GpuIndex(vecs, cols)
    bp = pred.concat([None] * 8, len(vecs))
    ids, dists, cnt, trunc = gi.brute_batch_raw(qs, bp, 300)
    o = cpu.exact_topk(vecs, cols, qs, bp, 300)
    check_exact(ids, dists, cnt, trunc, o[0], o[2], o[3], o[4], 300)


def test_non_integer_rows_within_tolerance():
    rng = np.random.default_rng(11)
    vecs = rng.standard_normal((20000, 64)).astype(np.float32)
    qs = rng.standard_normal((16, 64)).astype(np.float32)
    gi = GpuIndex(vecs, np.zeros((0, 20000)))
    bp = pred.concat([None] * 16, 20000)
    ids, dists, cnt, _ = gi.brute_batch_raw(qs, bp, 20)
    o_ids, o_d64 = cpu.exact_topk(vecs, np.zeros((0, 20000)), qs, bp, 20)[:2]
    for q in range(16):
        # distances within 1e-5 relative of the FP64 oracle, in order
        np.testing.assert_allclose(dists[q], o_d64[q], rtol=1e-5)
        exact = np.sum((vecs[ids[q].astype(np.int64)].astype(np.float64) - qs[q]) ** 2, 1)
        np.testing.assert_allclose(dists[q], exact, rtol=1e-5)
        # an id may differ only where the FP64 distances are within tolerance
        diff = ids[q] != o_ids[q]
        assert np.all(np.abs(o_d64[q][diff] - exact[diff]) <= 1e-5 * o_d64[q][diff])


def test_errors_leave_the_index_usable(golden_index, brute_golden):
    g = brute_golden
    q = g["queries"][:2]
    with pytest.raises(GpuError):
        golden_index.brute_batch(q, [None, None], 0)
    with pytest.raises(GpuError):
        golden_index.brute_batch(q, [None, None], 4097)
    with pytest.raises(GpuError):
        golden_index.brute_batch(np.zeros((1025, 128), np.float32), [None] * 1025, 10)
    bp = pred.concat([datagen.config1_predicate()] * 2, len(g["vectors"]))
    bp.qd["proot"][1] = 1000
    with pytest.raises(GpuError):
        golden_index.brute_batch_raw(q, bp, 10)
    ids, dists, cnt, trunc = golden_index.brute_batch(q, [None, None], 10)
    assert cnt.tolist() == [10, 10]


def test_prepared_batch_matches_abi(golden_index, brute_golden):
    import ctypes as C
    from paves_b200 import _lib
    g = brute_golden
    L = _lib.lib()
    nq = 16
    preds = [g["preds"][i % 5] for i in range(nq)]
    bp = pred.concat(preds, len(g["vectors"]))
    q = np.ascontiguousarray(g["queries"][:nq])
    err = C.create_string_buffer(256)
    b = L.pv_batch_create(golden_index.handle, nq, _lib.ptr(q), _lib.ptr(bp.qd),
                          _lib.ptr(bp.nodes), len(bp.nodes), _lib.ptr(bp.children),
                          len(bp.children), _lib.ptr(bp.invals), len(bp.invals), 10,
                          _lib.PV_MODE_EXACT, err, 256)
    assert b, err.value
    st = (C.c_float * 4)()
    tot = C.c_float()
    assert L.pv_batch_run(b, 3, st, C.byref(tot), err, 256) == 0
    assert tot.value > 0
    out = np.zeros(nq * 10, _lib.HIT_DTYPE)
    cnt = np.zeros(nq, np.uint32)
    tr = np.zeros(nq, np.uint8)
    assert L.pv_batch_fetch(b, _lib.ptr(out), _lib.ptr(cnt), _lib.ptr(tr), err, 256) == 0
    L.pv_batch_free(b)
    ids, dists, cnt2, tr2 = golden_index.brute_batch_raw(q, bp, 10)
    assert np.array_equal(out["node"].reshape(nq, 10), ids)
    assert np.array_equal(cnt, cnt2) and np.array_equal(tr, tr2)
