"""CPU oracle of the learned router (test infrastructure only).

No reference counterpart: the router is an addition beside the reference's
plain cost rule (extension/paves/src/planner.c:185-346, exec.c:415-424),
so this oracle is pinned by a finite-difference check of its own gradient
(tests/test_router_oracle.py) instead of reference fixtures.

Restates, in float64, what paves_b200/csrc/router.cu computes:
  * features: log10(selectivity), |q|, distances to the 8 nearest
    centroids, log2(k), predicate root kind;
  * a 12 -> 64 -> 64 -> 5 ReLU MLP whose forward multiplies by the
    bf16-rounded (round to nearest even) weights, inputs standardized by
    (x - mean) / std in float32;
  * the sample-weighted mean softmax cross-entropy and its gradient with
    respect to those effective weights.
"""
from __future__ import annotations

import numpy as np

NI, NH, NO = 12, 64, 5
SHAPES = [("W1", (NI, NH)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)),
          ("W3", (NH, NO)), ("b3", (NO,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return (r.astype(np.uint32) << 16).view(np.float32)


def unpack(params: np.ndarray):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(params[o:o + n], np.float64).reshape(shp)
        o += n
    return out


def pack(d) -> np.ndarray:
    return np.concatenate([np.asarray(d[n], np.float64).ravel() for n, _ in SHAPES])


def standardize(X, mean, std):
    X = np.asarray(X, np.float32)
    return ((X - np.asarray(mean, np.float32)) / np.asarray(std, np.float32)).astype(np.float64)


def forward_eff(w, Xn):
    """Forward with effective (already rounded) weights w (dict, float64)."""
    Z1 = Xn @ w["W1"] + w["b1"]
    H1 = np.maximum(Z1, 0.0)
    Z2 = H1 @ w["W2"] + w["b2"]
    H2 = np.maximum(Z2, 0.0)
    Z3 = H2 @ w["W3"] + w["b3"]
    return H1, H2, Z3


def logits(params, mean, std, X):
    w = unpack(bf16_round(np.asarray(params, np.float32)))
    return forward_eff(w, standardize(X, mean, std))[2]


def loss_eff(w, Xn, y, sw):
    Z3 = forward_eff(w, Xn)[2]
    m = Z3.max(1, keepdims=True)
    lse = np.log(np.exp(Z3 - m).sum(1)) + m[:, 0]
    ce = lse - Z3[np.arange(len(y)), y]
    return float((sw * ce).sum() / sw.sum())


def grad_eff(w, Xn, y, sw):
    """(loss, gradient dict) with respect to the effective weights."""
    H1, H2, Z3 = forward_eff(w, Xn)
    m = Z3.max(1, keepdims=True)
    e = np.exp(Z3 - m)
    p = e / e.sum(1, keepdims=True)
    W = sw.sum()
    onehot = np.zeros_like(p)
    onehot[np.arange(len(y)), y] = 1.0
    d3 = sw[:, None] * (p - onehot) / W
    d2 = (d3 @ w["W3"].T) * (H2 > 0)
    d1 = (d2 @ w["W2"].T) * (H1 > 0)
    g = {"W1": Xn.T @ d1, "b1": d1.sum(0), "W2": H1.T @ d2, "b2": d2.sum(0),
         "W3": H2.T @ d3, "b3": d3.sum(0)}
    ce = np.log(e.sum(1)) + m[:, 0] - Z3[np.arange(len(y)), y]
    return float((sw * ce).sum() / W), g


def grad(params, mean, std, X, y, sw=None):
    """(loss, flat gradient) as pv_router_grad defines them."""
    y = np.asarray(y, np.int64)
    sw = np.ones(len(y)) if sw is None else np.asarray(sw, np.float64)
    w = unpack(bf16_round(np.asarray(params, np.float32)))
    loss, g = grad_eff(w, standardize(X, mean, std), y, sw)
    return loss, pack(g)


def features(queries, centroids, sel, k, kind):
    """Router features [nq][12] (sel: selectivity per query in [0, 1])."""
    q = np.asarray(queries, np.float64)
    c = np.asarray(centroids, np.float64)
    d2 = (q * q).sum(1)[:, None] - 2.0 * q @ c.T + (c * c).sum(1)[None, :]
    d2 = np.maximum(d2, 0.0)
    near = np.sort(d2, 1)[:, :8]
    f = np.zeros((len(q), NI))
    f[:, 0] = np.log10(np.maximum(np.asarray(sel, np.float64), 1e-6))
    f[:, 1] = np.sqrt((q * q).sum(1))
    f[:, 2:10] = np.sqrt(near)
    f[:, 10] = np.log2(np.maximum(np.asarray(k, np.float64), 1))
    f[:, 11] = kind
    return f
