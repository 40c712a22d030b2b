"""Learned router kernels against the CPU oracle (oracle/mlp.py): features,
bf16 forward, gradients of the training step, and training itself."""
import numpy as np
import pytest

from oracle import mlp
from paves_b200 import GpuIndex, datagen, pred
from paves_b200.router import Router, init_params, kmeans

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    ds = datagen.make_dataset(20000, 64, nq=96)
    cent = kmeans(ds.vectors, 64, iters=4, sample=8192)
    g = GpuIndex(ds.vectors, ds.cols)
    r = Router(cent)
    yield ds, cent, g, r
    r.close()
    g.close()


def test_features_match_oracle(setup):
    ds, cent, g, r = setup
    kinds = list(datagen.six_predicates().values()) + [None]
    preds = [kinds[i % len(kinds)] for i in range(96)]
    ks = np.array([[1, 10, 100][i % 3] for i in range(96)], np.uint32)
    bp = pred.concat(preds, 20000)
    f = r.features(g, ds.queries, bp, ks)
    sel = np.array([pred.eval_numpy(p, ds.cols).mean() if p is not None else 1.0
                    for p in preds])
    kind = np.array([0 if p is None else {pred.Cmp: 1, pred.In: 2, pred.And: 3, pred.Or: 4,
                                            pred.Not: 5}[type(p)] for p in preds])
    ref = mlp.features(ds.queries, cent, sel, ks, kind)
    # selectivity is exact (bitmap popcount); distances in fp32
    assert np.allclose(f[:, 0], ref[:, 0], atol=1e-5)
    assert np.allclose(f[:, 1], ref[:, 1], rtol=1e-5)
    assert np.allclose(f[:, 2:10], ref[:, 2:10], rtol=1e-4, atol=1e-2)
    assert np.array_equal(f[:, 10:], ref[:, 10:].astype(np.float32))


def test_forward_and_gradient_match_oracle(setup):
    ds, cent, g, r = setup
    rng = np.random.default_rng(5)
    n = 777
    X = rng.standard_normal((n, 12)).astype(np.float32) * 3 + 2
    mean, std = X.mean(0), X.std(0)
    params = init_params(3)
    params[-5:] = rng.standard_normal(5).astype(np.float32) * 0.1
    r.set_params(params, mean, std)
    z = r.logits(X)
    zr = mlp.logits(params, mean, std, X)
    assert np.allclose(z, zr, rtol=1e-4, atol=1e-4)
    y = rng.integers(0, 5, n)
    sw = rng.uniform(0.2, 3.0, n).astype(np.float32)
    loss, gg = r.grad(X, y, sw)
    lr_, gr = mlp.grad(params, mean, std, X, y, sw)
    assert abs(loss - lr_) <= 1e-4 * max(1.0, abs(lr_))
    # ReLU gates sit at the same side in fp32 and fp64 except at exact
    # zeros; compare the whole vector by relative norm and per entry
    rel = np.linalg.norm(gg - gr) / np.linalg.norm(gr)
    assert rel < 1e-4, rel
    assert np.allclose(gg, gr, rtol=1e-3, atol=1e-6 * np.abs(gr).max())


def test_training_learns_a_separable_rule(setup):
    ds, cent, g, r = setup
    rng = np.random.default_rng(9)
    n = 16384
    X = rng.standard_normal((n, 12)).astype(np.float32)
    y = np.select([X[:, 0] > 0.8, X[:, 0] > 0, X[:, 1] > 0.5, X[:, 2] > 0], [1, 2, 3, 4], 0)
    r.set_params(init_params(1), X.mean(0), X.std(0))
    hist = r.train(X, y, epochs=30, batch=512, lr=3e-3)
    assert hist[-1] < 0.5 * hist[0]
    acc = (r.logits(X).argmax(1) == y).mean()
    assert acc > 0.95, acc
    # the weights that went through training still match the oracle forward
    p = r.params()
    assert np.allclose(r.logits(X[:256]), mlp.logits(p, X.mean(0), X.std(0), X[:256]),
                       rtol=1e-4, atol=1e-4)
