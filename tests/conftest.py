import hashlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _sha(*arrs):
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="session")
def brute_golden():
    """Dataset and reference BruteCursor results of tests/golden/brute_golden.npz."""
    from paves_b200 import datagen
    g = np.load(os.path.join(GOLDEN, "brute_golden.npz"))
    ds = datagen.make_dataset(20000, 128, nq=32)
    cols = ds.cols.copy()
    cols[datagen.COL_PRICE, ::int(g["nan_price_step"])] = np.nan
    cols[datagen.COL_CATEGORY, int(g["nan_cat_start"])::int(g["nan_cat_step"])] = np.nan
    assert _sha(ds.vectors, cols) == str(g["data_sha"]), "generator output changed"
    assert np.array_equal(ds.queries, g["queries"])
    from tests.golden_preds import brute_predicates
    return dict(vectors=ds.vectors, cols=cols, queries=ds.queries, preds=brute_predicates(),
                ids10=g["ids10"], d10=g["d10"], ids100=g["ids100"], d100=g["d100"])


@pytest.fixture(scope="session")
def graph_golden():
    from paves_b200 import datagen
    g = np.load(os.path.join(GOLDEN, "graph_golden.npz"))
    ds = datagen.make_dataset(4000, 128, nq=24)
    assert _sha(ds.vectors, ds.cols) == str(g["data_sha"]), "generator output changed"
    from tests.golden_preds import graph_predicates
    d = {k: g[k] for k in g.files}
    d.update(vectors=ds.vectors, cols=ds.cols, preds=graph_predicates())
    return d


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
