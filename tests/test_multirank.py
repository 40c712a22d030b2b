"""The multi-rank parts of bench.py on CPU: two gloo ranks share one HNSW
build through the host cache (rank 0 builds, the other loads after a
barrier) and reduce their timings to the maximum."""
import os
import socket
import tempfile

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, cache, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    from paves_b200 import datagen
    ds = datagen.make_dataset(1500, 16, nq=4)
    h = bench.shared_graph(ds.vectors, rank, dist, cache)
    mx = bench.reduce_max([float(rank + 1), 10.0 - rank], dist, "cpu")
    np.savez(os.path.join(out, f"r{rank}.npz"), l0=h.l0, entry=h.entry_node, mx=np.array(mx))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_share_graph_and_max_time():
    with tempfile.TemporaryDirectory() as td:
        cache = os.path.join(td, "g.npz")
        mp.start_processes(_rank, args=(2, _free_port(), cache, td), nprocs=2, join=True,
                           start_method="spawn")
        a, b = (np.load(os.path.join(td, f"r{r}.npz")) for r in range(2))
        assert np.array_equal(a["l0"], b["l0"]) and int(a["entry"]) == int(b["entry"])
        assert a["mx"].tolist() == b["mx"].tolist() == [2.0, 10.0]
        assert os.path.exists(cache)
