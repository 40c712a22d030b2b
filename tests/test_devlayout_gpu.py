"""Stored device layout through the C ABI: an index's low-precision rows,
norms and scales are read back, stored beside its index file, read again
and uploaded as straight copies; the new index holds byte-identical device
arrays and answers every batch exactly as the converted one."""
import os
import tempfile

import numpy as np
import pytest

from paves_b200 import GpuIndex, _lib, datagen, pred
from paves_b200.hnsw import Hnsw
from paves_b200.indexfile import read_device_layout, read_index, write_device_layout

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [_lib.FV_GPU_PREC_BF16, _lib.FV_GPU_PREC_FP8])
def test_prepared_upload_matches_converted(prec):
    n, d = 30_011, 96
    ds = datagen.make_dataset(n, d, nq=40)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "idx.pvf")
        Hnsw(ds.vectors, 4, 16).write(path, ds.cols)
        f = read_index(path)
        gi = GpuIndex(f.vectors, f.cols, precision=prec)
        lay = gi.export_device_layout()
        write_device_layout(path, lay)
        back = read_device_layout(path, prec)
        assert back is not None
        gi2 = GpuIndex(f.vectors, f.cols, precision=prec, prepared=back)
        lay2 = gi2.export_device_layout()
        assert lay2.row_amax == lay.row_amax and lay2.kpad == lay.kpad
        assert np.array_equal(lay2.rows, lay.rows) and np.array_equal(lay2.norms, lay.norms)
        if prec == _lib.FV_GPU_PREC_FP8:
            assert np.array_equal(lay2.scales, lay.scales)
        six = list(datagen.six_predicates().values()) + [None]
        preds = [six[q % len(six)] for q in range(40)]
        bp = pred.concat(preds, n)
        for topb in (1, 10):
            a = gi.brute_batch_raw(ds.queries, bp, topb)
            sa = _lib.lib().pv_last_superset(gi.handle)
            b = gi2.brute_batch_raw(ds.queries, bp, topb)
            assert _lib.lib().pv_last_superset(gi2.handle) == sa
            for x, y in zip(a, b):
                assert np.array_equal(x, y)
        gi2.close()
        gi.close()
