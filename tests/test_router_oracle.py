"""Pins the router's CPU oracle (oracle/mlp.py): its analytic gradient
against central finite differences in float64, and its bf16 rounding
against exhaustive properties. CPU only."""
import numpy as np

from oracle import mlp


def _setup(seed=3, n=40):
    rng = np.random.default_rng(seed)
    params = (rng.standard_normal(mlp.NPARAMS) * 0.3).astype(np.float32)
    X = rng.standard_normal((n, mlp.NI)).astype(np.float32) * 2 + 1
    mean = X.mean(0)
    std = X.std(0) + 0.1
    y = rng.integers(0, mlp.NO, n)
    sw = rng.uniform(0.5, 2.0, n)
    return params, X, mean, std, y, sw


def test_gradient_matches_finite_differences():
    params, X, mean, std, y, sw = _setup()
    w = mlp.unpack(mlp.bf16_round(params))
    Xn = mlp.standardize(X, mean, std)
    loss, g = mlp.grad_eff(w, Xn, y, sw)
    assert abs(loss - mlp.loss_eff(w, Xn, y, sw)) < 1e-12
    rng = np.random.default_rng(0)
    h = 1e-6
    for name, shp in mlp.SHAPES:
        flat = w[name].reshape(-1)
        for idx in rng.choice(flat.size, min(12, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp = mlp.loss_eff(w, Xn, y, sw)
            flat[idx] = old - h
            lm = mlp.loss_eff(w, Xn, y, sw)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            an = g[name].reshape(-1)[idx]
            assert abs(fd - an) <= 1e-6 + 1e-5 * abs(fd), (name, idx, fd, an)


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.14159, 0.0, 65504.0], np.float32)
    r = mlp.bf16_round(x)
    # every result is a bf16 value (low 16 bits zero) within half an ulp
    assert (r.view(np.uint32) & 0xFFFF == 0).all()
    ulp = np.abs(x) * 2.0 ** -7
    assert (np.abs(r - x) <= ulp / 2 + 1e-30).all()
    # ties go to the even mantissa: 1 + 2^-8 lies halfway between 1 and 1 + 2^-7
    assert r[1] == 1.0
    assert r[3] == np.float32(1.0078125)


def test_features_shape_and_order():
    rng = np.random.default_rng(1)
    q = rng.integers(0, 255, (5, 16)).astype(np.float32)
    c = rng.integers(0, 255, (20, 16)).astype(np.float32)
    f = mlp.features(q, c, [1.0, 0.5, 0.01, 1e-9, 0.3], [10, 1, 100, 10, 7], [0, 1, 2, 3, 4])
    assert f.shape == (5, 12)
    assert (np.diff(f[:, 2:10], axis=1) >= 0).all()
    assert f[3, 0] == -6.0 and f[0, 0] == 0.0
    assert np.allclose(f[:, 10], np.log2([10, 1, 100, 10, 7]))
