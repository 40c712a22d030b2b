"""The tensor-core scan's bounded waits, made to run out on purpose.

Every wait of scan_tc_kernel (TMA stages, MMA completion, tensor-memory
buffers, the norm ring) gives up at a deadline; the kernel then records
which role gave up, waits (with its own, separate 2 s limit) for the copies
and MMAs it already issued, frees its tensor memory and returns. Here the
limit is set to 1 ns, so the first wait that is not already over expires: the batch call must return
-1 with the error message, nothing may fault or hang, and with the default
limit restored the same index must answer a batch exactly (oracle)."""
import numpy as np
import pytest

from oracle import cpu
from paves_b200 import GpuError, GpuIndex, _lib, datagen, pred

pytestmark = pytest.mark.gpu


def test_expired_waits_return_an_error_and_the_index_still_serves():
    ds = datagen.make_dataset(300_000, 128, nq=64)
    gi = GpuIndex(ds.vectors, ds.cols, precision=_lib.FV_GPU_PREC_BF16)
    L = _lib.lib()
    preds = [list(datagen.six_predicates().values())[2 + q % 4] for q in range(64)]
    gi.brute_batch(ds.queries, preds, 10)  # warm: scratch sized, kernels loaded
    assert L.pv_tc_timeout(gi.handle, 1) == 0  # 1 ns: every wait that must wait expires
    for _ in range(3):
        with pytest.raises(GpuError, match="wait expired"):
            gi.brute_batch(ds.queries, preds, 10)
    assert L.pv_tc_timeout(gi.handle, 0) == 0
    assert L.pv_tc_timeout(gi.handle, 20_000_000_000) == -1  # over 10 s
    ids, dists, cnt, trunc = gi.brute_batch(ds.queries, preds, 10)
    bp = pred.concat(preds, len(ds.vectors))
    o_ids, _, o_d32, o_cnt, _ = cpu.exact_topk(ds.vectors, ds.cols, ds.queries, bp, 10)
    assert np.array_equal(cnt, o_cnt)
    for q in range(64):
        n = int(cnt[q])
        assert np.array_equal(ids[q, :n], o_ids[q, :n].astype(np.uint64)), q
        assert np.array_equal(dists[q, :n], o_d32[q, :n]), q
    gi.close()
