"""Row shards on the GPU: an index split into 2 and 3 row shards (each a
GpuIndex through the C ABI) merges to exactly the answer of one index
holding every row: ids and FP32 distances bit-identical, counts and
truncation flags equal."""
import numpy as np
import pytest

from paves_b200 import GpuIndex, datagen, pred
from paves_b200.shard import LocalShards

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nshards", [2, 3])
def test_row_shards_merge_to_the_whole_index_answer(nshards):
    n = 50_001
    ds = datagen.make_dataset(n, 64, nq=24)
    six = list(datagen.six_predicates().values()) + [None]
    preds = [six[q % len(six)] for q in range(24)]
    whole = GpuIndex(ds.vectors, ds.cols)
    shards = LocalShards(ds.vectors, ds.cols, nshards)
    for topb in (1, 10, 256):
        w_ids, w_d, w_c, w_t = whole.brute_batch(ds.queries, preds, topb)
        s_ids, s_d, s_c, s_t = shards.brute_batch(ds.queries, preds, topb)
        assert np.array_equal(w_c, s_c) and np.array_equal(w_t, s_t)
        for q in range(24):
            c = int(w_c[q])
            assert np.array_equal(w_ids[q, :c], s_ids[q, :c]), (topb, q)
            assert np.array_equal(w_d[q, :c], s_d[q, :c]), (topb, q)
    shards.close()
    whole.close()
