"""Host-side logic that needs no GPU: the C-ABI library loads and exports
every declared symbol, predicate serialization matches the reference's,
host predicate validation, the index file format."""
import ctypes as C
import os
import re
import tempfile

import numpy as np
import pytest

from paves_b200 import _lib, datagen, pred
from paves_b200.indexfile import read_index, write_index

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b((?:fv|pv)_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    decl = declared_functions()
    assert len(decl) >= 16
    for name in decl:
        assert hasattr(L, name), name
    assert set(_lib.exported_symbols()) == decl


def test_struct_layouts():
    assert C.sizeof(_lib.FvGpuPredNode) == 40
    assert C.sizeof(_lib.FvGpuQueryDesc) == 32
    assert C.sizeof(_lib.FvHit) == 16
    assert C.sizeof(_lib.FvGpuSpan) == 12


def _check(bp, ncols=2):
    L = _lib.lib()
    err = C.create_string_buffer(256)
    nprog = C.c_int(0)
    rc = L.pv_pred_check(len(bp.qd), _lib.ptr(bp.qd), _lib.ptr(bp.nodes), len(bp.nodes),
                         _lib.ptr(bp.children), len(bp.children), _lib.ptr(bp.invals),
                         len(bp.invals), ncols, C.byref(nprog), err, 256)
    return rc, nprog.value, err.value.decode()


def test_pred_check_dedupes_identical_predicates():
    p1 = datagen.config1_predicate()
    p2 = datagen.config1_predicate()  # equal tree, separate object
    p3 = pred.Cmp(1, "<", 5.0)
    bp = pred.concat([p1, p2, None, p3, p1], 100)
    rc, nprog, _ = _check(bp)
    assert rc == 0 and nprog == 2


@pytest.mark.parametrize("mutate,msg", [
    (lambda bp: bp.qd.__setitem__(("proot"), np.int32(99)), "out of range"),
    (lambda bp: bp.nodes.__setitem__(("col"), 7), "column out of range"),
    (lambda bp: bp.children.__setitem__(0, 50), "out of range"),
    (lambda bp: bp.nodes.__setitem__(("kind"), 9), "unknown"),
])
def test_pred_check_rejects_bad_arrays(mutate, msg):
    bp = pred.concat([datagen.config1_predicate()], 100)
    mutate(bp)
    rc, _, err = _check(bp)
    assert rc == -1 and msg in err


def test_pred_check_rejects_cycles():
    bp = pred.concat([pred.And(pred.Cmp(0, "<", 1.0), pred.Cmp(1, "<", 1.0))], 100)
    bp.children[0] = 0  # AND's first child is itself
    rc, _, err = _check(bp)
    assert rc == -1


def test_wide_and_is_folded():
    # 90 conjuncts (the arbiter slot allows 96 children): folded to binary
    # steps, so the evaluation stack stays shallow
    p = pred.And(*[pred.Cmp(1, ">", float(-i)) for i in range(90)])
    rc, nprog, err = _check(pred.concat([p], 10))
    assert rc == 0, err


@pytest.mark.skipif(not __import__("oracle.refengine").refengine.available("cpu"),
                    reason="reference engine not built")
def test_serialize_matches_reference_fv_pred_serialize():
    from oracle import refengine
    ds = datagen.make_dataset(500, 16, nq=1)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "s.idx")
        refengine.build_index(path, ds.vectors, ds.cols, M=4, efc=8)
        R = refengine.RefIndex(path)
        L = R.L
        for p in [datagen.config1_predicate(),
                  pred.Or(pred.Not(pred.In(0, [1, 2, 3])), pred.Cmp(1, "!=", 3.5),
                          pred.And(pred.Cmp(1, ">=", 1.0), pred.Cmp(1, "<", 9.0)))]:
            ph = R.compile(p)
            nodes = np.zeros(64, _lib.NODE_DTYPE)
            children = np.zeros(64, np.int32)
            invals = np.zeros(64, np.float64)
            spans = np.zeros(64, _lib.SPAN_DTYPE)
            bpc = refengine.FvGpuBatchPred()
            total = C.c_uint64(0)
            rc = L.fv_pred_serialize(R.h, ph, nodes.ctypes.data, 64, children.ctypes.data, 64,
                                     invals.ctypes.data, 64, spans.ctypes.data, 64,
                                     C.byref(bpc), C.byref(total))
            assert rc == 0
            s = pred.serialize(p)
            assert bpc.nnodes == len(s.nodes)
            assert np.array_equal(nodes[:bpc.nnodes], s.nodes)
            assert np.array_equal(children[:bpc.nchildren], s.children)
            assert np.array_equal(invals[:bpc.ninvals], s.invals)
            R.free_pred(ph)
        R.close()


def test_index_file_roundtrip():
    rng = np.random.default_rng(1)
    n, d, M = 300, 8, 4
    vecs = rng.integers(0, 255, (n, d)).astype(np.float32)
    cols = rng.uniform(0, 10, (2, n))
    cols[1, ::7] = np.nan
    stride = 2 * M + 1
    l0 = np.zeros((n, stride), np.uint32)
    l0[:, 0] = 3
    l0[:, 1:4] = rng.integers(0, n, (n, 3))
    levels = np.zeros(n, np.uint8)
    levels[5] = 2
    uoffs = np.zeros(n + 1, np.uint64)
    uoffs[6:] = 2 * (M + 1)
    upper = np.zeros(2 * (M + 1), np.uint32)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "w.idx")
        write_index(path, vecs, cols, M, 32, levels, l0, uoffs, upper, max_level=2,
                    entry_node=5)
        f = read_index(path)
        assert f.count == n and f.dim == d and f.M == M and f.entry_node == 5
        assert np.array_equal(f.vectors, vecs)
        assert np.array_equal(f.cols, cols, equal_nan=True)
        assert np.array_equal(f.l0, l0)
        # posting lists: NaN last, ties by row
        v = f.post_vals[1]
        fin = ~np.isnan(v)
        assert fin[: fin.sum()].all() and np.all(np.diff(v[fin]) >= 0)
        from oracle import refengine
        if refengine.available("cpu"):
            R = refengine.RefIndex(path)  # the reference engine opens our file
            assert R.graph_entry(vecs[0]) in range(n)
            R.close()


def test_identical_predicate_trees_share_one_program():
    """Batches carry one serialized tree per query; structurally identical
    trees (any slice of the arrays) compile to one program, as do trees whose
    compiled programs are equal; distinct ones (down to a constant's bits:
    -0.0 vs 0.0) stay apart, and a malformed tree is still reported."""
    import ctypes as C
    from paves_b200 import _lib, pred
    L = _lib.lib()
    P, Cc = 0, 1

    def nprog(preds, ncols=2):
        bp = pred.concat(preds, 100)
        err = C.create_string_buffer(256)
        n = C.c_int()
        rc = L.pv_pred_check(len(preds), _lib.ptr(bp.qd), _lib.ptr(bp.nodes), len(bp.nodes),
                             _lib.ptr(bp.children), len(bp.children), _lib.ptr(bp.invals),
                             len(bp.invals), ncols, C.byref(n), err, 256)
        return rc, n.value, err.value

    a = pred.And(pred.Cmp(P, "<", 10.0), pred.In(Cc, [3.0, 7.0]))
    b = pred.Or(pred.Cmp(P, ">", 5.0), pred.Not(pred.In(Cc, [1.0])))
    assert nprog([a] * 64)[:2] == (0, 1)
    assert nprog([a, None, b] * 21)[:2] == (0, 2)
    assert nprog([pred.Cmp(P, "==", 0.0), pred.Cmp(P, "==", -0.0)] * 8)[:2] == (0, 2)
    # different trees that compile to the same program (one integer set) share it
    assert nprog([pred.In(Cc, [1.0, 2.0]), pred.In(Cc, [2.0, 1.0])])[:2] == (0, 1)
    rc, _, msg = nprog([a, pred.Cmp(5, "<", 1.0)])  # column 5 of 2
    assert rc == -1 and b"column" in msg
