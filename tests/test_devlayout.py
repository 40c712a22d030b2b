"""The stored device layout beside an index file (no GPU): round trip of
the companion file, and the checks that make a loader fall back to
converting - another precision, an index file rewritten since, a
truncated or mis-strided companion."""
import os
import tempfile

import numpy as np
import pytest

from paves_b200 import datagen
from paves_b200.hnsw import Hnsw
from paves_b200.indexfile import (DeviceLayout, device_layout_path, read_device_layout,
                                  read_index, write_device_layout)

BF16, FP8 = 2, 3


def _index(td, n=300, d=20):
    ds = datagen.make_dataset(n, d, nq=2)
    path = os.path.join(td, "idx.pvf")
    Hnsw(ds.vectors, 4, 16).write(path, ds.cols)
    return path, ds


def _layout(prec, n, d, rng):
    kpad = (d + 127) & ~127 if prec == FP8 else (d + 63) & ~63
    esz = 1 if prec == FP8 else 2
    return DeviceLayout(prec, n, d, kpad, 37.0,
                        rng.integers(0, 256, n * kpad * esz, dtype=np.uint8),
                        rng.random(n, dtype=np.float32),
                        rng.random(n, dtype=np.float32) if prec == FP8 else None)


@pytest.mark.parametrize("prec", [BF16, FP8])
def test_round_trip(prec):
    rng = np.random.default_rng(1)
    with tempfile.TemporaryDirectory() as td:
        path, ds = _index(td)
        lay = _layout(prec, 300, 20, rng)
        write_device_layout(path, lay)
        back = read_device_layout(path, prec)
        assert back is not None and back.kpad == lay.kpad and back.row_amax == 37.0
        assert np.array_equal(back.rows, lay.rows) and np.array_equal(back.norms, lay.norms)
        if prec == FP8:
            assert np.array_equal(back.scales, lay.scales)
        else:
            assert back.scales is None
        assert read_index(path).count == 300  # the index file itself is untouched


def test_fallbacks_and_errors():
    rng = np.random.default_rng(2)
    with tempfile.TemporaryDirectory() as td:
        path, ds = _index(td)
        assert read_device_layout(path, FP8) is None  # none stored
        write_device_layout(path, _layout(FP8, 300, 20, rng))
        assert read_device_layout(path, BF16) is None  # stored for another precision
        # a rewritten index file (another graph: other offsets) makes it stale
        Hnsw(ds.vectors[:250], 4, 16).write(path, ds.cols[:, :250])
        assert read_device_layout(path, FP8) is None
        # the same count, dim and M with other vectors: node levels hash the
        # row number, so the header is byte-identical; the rows are not
        write_device_layout(path, _layout(FP8, 250, 20, rng))
        assert read_device_layout(path, FP8) is not None
        hdr0 = open(path, "rb").read(264)
        other = np.ascontiguousarray(ds.vectors[:250][::-1])
        Hnsw(other, 4, 16).write(path, ds.cols[:, :250])
        assert open(path, "rb").read(264) == hdr0
        assert read_device_layout(path, FP8) is None
        # matching but truncated
        write_device_layout(path, _layout(FP8, 250, 20, rng))
        dp = device_layout_path(path)
        with open(dp, "r+b") as f:
            f.truncate(os.path.getsize(dp) - 64)
        with pytest.raises(ValueError):
            read_device_layout(path, FP8)
        # arrays that do not match count / stride are refused at write time
        bad = _layout(FP8, 250, 20, rng)
        bad.rows = bad.rows[:-1]
        with pytest.raises(ValueError):
            write_device_layout(path, bad)
