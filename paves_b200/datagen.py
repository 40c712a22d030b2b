"""Seeded synthetic workloads.

The reference benchmarks on SIFT1M, which is not available here. These
generators stand in for it with the same shape and value distribution:
rows drawn from a Gaussian mixture (centres U[0,128]^d, sigma 20), clipped
to [0,255] and rounded to integers, stored as float32 -- integer-valued
like SIFT descriptors. Queries come from the same mixture on a separate
random stream and are never index rows. Attributes: ``category`` integer
uniform 0..9 and ``price`` float32 uniform [0,1000), stored as float64
column slots 0 and 1 like the engine's scalar columns.

Seed convention: ``numpy.random.default_rng(20240617 + stream)``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .pred import And, Cmp, In

SEED = 20240617
COL_CATEGORY, COL_PRICE = 0, 1


@dataclass
class Dataset:
    vectors: np.ndarray   # [N, d] float32
    cols: np.ndarray      # [2, N] float64 (category, price)
    queries: np.ndarray   # [nq, d] float32
    centers: np.ndarray   # [ncomp, d] float32


def _mixture(rng, centers, n, d, chunk=1 << 18):
    out = np.empty((n, d), np.float32)
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        comp = rng.integers(0, len(centers), m)
        x = rng.standard_normal((m, d), dtype=np.float32)
        x *= 20.0
        x += centers[comp]
        np.clip(x, 0.0, 255.0, out=x)
        np.rint(x, out=x)
        out[s:s + m] = x
    return out


def make_dataset(n: int, d: int = 128, nq: int = 256, ncomp: int = 64,
                 seed: int = SEED) -> Dataset:
    rng_c = np.random.default_rng(seed + 0)
    centers = rng_c.uniform(0.0, 128.0, (ncomp, d)).astype(np.float32)
    vectors = _mixture(np.random.default_rng(seed + 1), centers, n, d)
    queries = _mixture(np.random.default_rng(seed + 2), centers, nq, d)
    rng_a = np.random.default_rng(seed + 3)
    category = rng_a.integers(0, 10, n).astype(np.float64)
    price = rng_a.uniform(0.0, 1000.0, n).astype(np.float32).astype(np.float64)
    cols = np.stack([category, price])
    return Dataset(vectors, cols, queries, centers)


def make_queries(centers: np.ndarray, nq: int, seed: int = SEED, stream: int = 2):
    return _mixture(np.random.default_rng(seed + stream), centers, nq, centers.shape[1])


def posting_rows(cols: np.ndarray) -> np.ndarray:
    """Per column, row ids sorted by value (NaN last, ties by row id) --
    the posting lists fv_builder_finish writes (engine.cpp:921-941)."""
    out = np.empty(cols.shape, np.uint32)
    for c in range(cols.shape[0]):
        out[c] = np.argsort(cols[c], kind="stable").astype(np.uint32)
    return out


# Predicate kinds of the 1M x 128 configuration with their target
# selectivities (fraction of rows passing).
def six_predicates():
    return {
        "sel0.1%": And(Cmp(COL_PRICE, "<", 10.0), Cmp(COL_CATEGORY, "==", 3.0)),
        "sel1%": Cmp(COL_PRICE, "<", 10.0),
        "sel10%": In(COL_CATEGORY, [3]),
        "sel30%": In(COL_CATEGORY, [1, 4, 7]),
        "sel70%": Cmp(COL_PRICE, "<", 700.0),
        "sel95%": Cmp(COL_PRICE, "<", 950.0),
    }


def config1_predicate():
    """price < 100 AND category IN (3, 7): about 2% of rows."""
    return And(Cmp(COL_PRICE, "<", 100.0), In(COL_CATEGORY, [3, 7]))


def graph_predicates():
    """Bitmaps at 1%, 10% and 50% for the graph-search configuration."""
    return {
        "sel1%": Cmp(COL_PRICE, "<", 10.0),
        "sel10%": In(COL_CATEGORY, [3]),
        "sel50%": Cmp(COL_PRICE, "<", 500.0),
    }
