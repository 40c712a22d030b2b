"""The no-allocation entry point (pv_brute_batch_noalloc).

It serves callers that must not allocate device memory while answering
queries (an allocation synchronizes the device; some hosts own all device
memory). It takes device buffers from the caller and keeps its scratch in a
fixed array inside the library. Here it must return exactly what the
regular entry point (fv_gpu_brute_batch, no predicate) returns, on two
calls in a row with different queries, so nothing leaks from one call into
the next through the shared scratch.

This file sorts last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from paves_b200 import GpuIndex, _lib, datagen

pytestmark = pytest.mark.gpu


def _noalloc(gi, queries, topb):
    import torch
    L = _lib.lib()
    nq = queries.shape[0]
    dev = torch.device(f"cuda:{gi.device()}")
    d_q = torch.from_numpy(np.ascontiguousarray(queries, np.float32)).to(dev)
    d_out = torch.zeros(nq * topb * 16, dtype=torch.uint8, device=dev)
    d_cnt = torch.zeros(nq, dtype=torch.int32, device=dev)
    torch.cuda.synchronize(dev)
    err = C.create_string_buffer(256)
    rc = L.pv_brute_batch_noalloc(gi.handle, nq, d_q.data_ptr(), topb, d_out.data_ptr(),
                                  d_cnt.data_ptr(), err, 256)
    assert rc == 0, err.value.decode()
    out = d_out.cpu().numpy().view(_lib.HIT_DTYPE).reshape(nq, topb)
    return out["node"], out["dist"], d_cnt.cpu().numpy().astype(np.uint32)


def _compare(gi, queries, topb):
    ids, dists, cnt = _noalloc(gi, queries, topb)
    r_ids, r_dists, r_cnt, _ = gi.brute_batch(queries, [None] * len(queries), topb)
    assert np.array_equal(cnt, r_cnt)
    for q in range(len(queries)):
        n = int(r_cnt[q])
        assert np.array_equal(ids[q, :n], r_ids[q, :n]), q
        assert np.array_equal(dists[q, :n], r_dists[q, :n]), q


@pytest.mark.parametrize("dim", [128, 100])
def test_noalloc_matches_regular_entry_point_twice(dim):
    ds = datagen.make_dataset(120_001, dim, nq=40)
    gi = GpuIndex(ds.vectors, ds.cols, device=0)
    _compare(gi, ds.queries[:32], 32)   # first call: sets up the scratch address
    _compare(gi, ds.queries[8:20], 10)  # second call: different shape, shared scratch
    gi.close()


def test_noalloc_leaves_free_device_memory_unchanged():
    """The point of the entry point: after its first call on a device,
    further calls of any allowed shape allocate nothing on the device (the
    caller's buffers are allocated once, up front, at the largest shape)."""
    import torch
    ds = datagen.make_dataset(50_000, 96, nq=32)
    gi = GpuIndex(ds.vectors, ds.cols, device=0)
    dev = torch.device(f"cuda:{gi.device()}")
    L = _lib.lib()
    err = C.create_string_buffer(256)
    d_q = torch.from_numpy(np.ascontiguousarray(ds.queries, np.float32)).to(dev)
    d_out = torch.zeros(32 * 32 * 16, dtype=torch.uint8, device=dev)
    d_cnt = torch.zeros(32, dtype=torch.int32, device=dev)
    torch.cuda.synchronize(dev)

    def call(nq, topb):
        rc = L.pv_brute_batch_noalloc(gi.handle, nq, d_q.data_ptr(), topb, d_out.data_ptr(),
                                      d_cnt.data_ptr(), err, 256)
        assert rc == 0, err.value.decode()

    call(32, 32)  # first call on the device: looks up the scratch address
    free0, _ = torch.cuda.mem_get_info(dev)
    for nq, topb in [(1, 1), (32, 32), (7, 10), (16, 3), (32, 1), (2, 32)]:
        call(nq, topb)
        assert torch.cuda.mem_get_info(dev)[0] == free0, (nq, topb)
    # and the last call's answer is still the regular entry point's
    out = d_out.cpu().numpy()[:2 * 32 * 16].view(_lib.HIT_DTYPE).reshape(2, 32)
    r_ids, r_dists, r_cnt, _ = gi.brute_batch(ds.queries[:2], [None, None], 32)
    assert np.array_equal(out["node"], r_ids) and np.array_equal(out["dist"], r_dists)
    gi.close()


def test_noalloc_rejects_oversize_requests():
    ds = datagen.make_dataset(5000, 64, nq=40)
    gi = GpuIndex(ds.vectors, ds.cols, device=0)
    L = _lib.lib()
    err = C.create_string_buffer(256)
    rc = L.pv_brute_batch_noalloc(gi.handle, 33, 1, 10, 1, 1, err, 256)  # never dereferenced
    assert rc == -1 and b"nq <= 32" in err.value
    rc = L.pv_brute_batch_noalloc(gi.handle, 4, 1, 33, 1, 1, err, 256)
    assert rc == -1 and b"topb <= 32" in err.value
    gi.close()
