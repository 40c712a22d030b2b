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


def _bound(g, p):
    import ctypes as C
    from paves_b200 import _lib
    s = pred.serialize(p)
    b = C.c_uint64()
    err = C.create_string_buffer(256)
    rc = _lib.lib().pv_filter_bound(g.handle, _lib.ptr(s.nodes), len(s.nodes),
                                    _lib.ptr(s.children), len(s.children), _lib.ptr(s.invals),
                                    len(s.invals), C.byref(b), err, 256)
    assert rc == 0, err.value
    return int(b.value)


def test_selective_filters_take_the_sparse_route():
    """A batch sharing one selective filter scans only its matching rows
    (bitmap -> row list -> exact scan of the list); results equal the
    oracle's, and the host bound on matches never falls below the truth,
    including NaN attributes, NE, NOT, OR and duplicate IN values."""
    from paves_b200 import _lib
    rng = np.random.default_rng(11)
    n = 120_000
    ds = datagen.make_dataset(n, 64, nq=40)
    cols = ds.cols.copy()
    cols[1, rng.choice(n, 500, replace=False)] = np.nan
    g = GpuIndex(ds.vectors, cols)
    P, Cc = datagen.COL_PRICE, datagen.COL_CATEGORY
    preds = [pred.Cmp(P, "<", 5.0), pred.And(pred.Cmp(P, "<", 50.0), pred.In(Cc, [3.0, 3.0])),
             pred.Cmp(P, "==", float(cols[1][7])), pred.Not(pred.Cmp(P, ">=", 3.0)),
             pred.Or(pred.Cmp(P, "<", 2.0), pred.Cmp(P, ">", 998.0)),
             pred.And(pred.Cmp(P, "!=", 500.0), pred.Cmp(P, "<", 30.0)),
             pred.Cmp(P, "<", 600.0), pred.In(Cc, [1.0, 2.0])]
    routes = []
    for p in preds:
        truth = int(pred.eval_numpy(p, cols).sum())
        assert _bound(g, p) >= truth, p
        for topb in (1, 10, 300):
            ids, dists, cnt, trunc = g.brute_batch(ds.queries, [p] * 40, topb)
            routes.append(_lib.lib().pv_last_sparse(g.handle))
            bp = pred.concat([p] * 40, n)
            o = cpu.exact_topk(ds.vectors, cols, ds.queries, bp, topb)
            check_exact(ids, dists, cnt, trunc, o[0], o[2], o[3], o[4], topb)
    assert sum(routes) >= 15 and min(routes) == 0  # selective ones sparse, broad ones dense
    g.close()


def test_range_form_edge_values():
    """Programs that are ANDs of comparisons and IN lists run in range form
    (per-column intervals, small-integer sets); the rest on the bit-stack
    interpreter. Both in one batch (one predicate per query, several
    program chunks), over attributes holding NaN, +-inf, -0.0, half
    integers and the 63/64 set boundary, against the oracle's match sets;
    the host bound never falls below the oracle's count."""
    rng = np.random.default_rng(5)
    n = 4000
    ds = datagen.make_dataset(n, 16, nq=1)
    edge0 = np.array([np.nan, np.inf, -np.inf, -0.0, 0.0, 1.0, 62.0, 63.0, 63.5, 64.0, 65.0,
                      -1.0, 1e300, -1e300, 5e-324, 3.0, 2.9999999999999996])
    edge1 = np.array([np.nan, -0.0, 0.0, 1.0, 2.0, 3.0, 4.0, 9.0, 63.0, 64.0, 2.5, -3.0])
    cols = np.empty((2, n))
    cols[0] = np.where(rng.random(n) < 0.5, rng.choice(edge0, n), rng.integers(0, 100, n))
    cols[1] = np.where(rng.random(n) < 0.5, rng.choice(edge1, n), rng.integers(0, 10, n))
    g = GpuIndex(ds.vectors, cols)
    C_, I_, A_ = pred.Cmp, pred.In, pred.And
    consts = [np.nan, np.inf, -np.inf, -0.0, 0.0, 63.0, 63.5, 64.0, 3.0]
    preds = [C_(c, op, v) for c in (0, 1) for op in ("<", "<=", ">", ">=", "==", "!=")
             for v in consts]
    preds += [
        A_(C_(0, ">=", 3.0), C_(0, "<", 64.0)), A_(C_(0, ">", 3.0), C_(0, ">=", 3.0)),
        A_(C_(0, "<=", 63.0), C_(0, "<", 63.0)), A_(C_(0, "==", np.nan), C_(0, "<", 5.0)),
        A_(C_(0, ">", -np.inf), C_(0, "<", np.inf)), A_(C_(0, ">=", 64.0), C_(0, "<=", 3.0)),
        A_(I_(1, [1.0, 2.0, 3.0]), I_(1, [2.0, 3.0, 4.0])),
        A_(I_(1, [63.0, 0.0]), C_(0, "<", 100.0)), A_(), I_(1, []), I_(1, [2.5]),
        I_(1, [2.5, 2.5]), I_(1, [2.5, 3.0]), I_(1, [-0.0]), I_(1, [64.0]), I_(0, [np.nan]),
        I_(0, [63.0, 64.0]), A_(A_(C_(0, ">=", 1.0), I_(1, [1.0, 9.0])),
                                  A_(C_(0, "<=", 62.0), C_(1, "<", 9.0))),
        A_(C_(0, ">=", 0.0), C_(0, "<=", -0.0)), A_(I_(1, [3.0]), C_(1, ">=", 3.0)),
        pred.Or(C_(0, "<", 1.0), C_(1, "==", 2.0)), pred.Not(C_(0, "<", 3.0)),
        A_(C_(0, "<", 50.0), pred.Not(I_(1, [2.0]))), A_(C_(0, "!=", 3.0), C_(0, "<", 10.0)),
    ]
    nq = len(preds)
    q = np.repeat(ds.queries[:1], nq, axis=0)
    ids, dists, cnt, trunc = g.brute_batch(q, preds, 4096)
    bp = pred.concat(preds, n)
    o = cpu.exact_topk(ds.vectors, cols, q, bp, 4096)
    check_exact(ids, dists, cnt, trunc, o[0], o[2], o[3], o[4], 4096)
    for i, p in enumerate(preds):
        assert _bound(g, p) >= int(o[4][i]), p
    # each predicate alone: a batch sharing one range-form filter takes the
    # lean bitmap kernel, the others the general one; both as the oracle
    for i, p in enumerate(preds):
        q2 = np.repeat(ds.queries[:1], 2, axis=0)
        ids2, dists2, cnt2, trunc2 = g.brute_batch(q2, [p, p], 4096)
        for j in range(2):
            check_exact(ids2[j:j + 1], dists2[j:j + 1], cnt2[j:j + 1], trunc2[j:j + 1],
                        o[0][i:i + 1], o[2][i:i + 1], o[3][i:i + 1], o[4][i:i + 1], 4096)
    g.close()
