"""Multi-process (world_size 2, gloo on CPU) test of the chain sharding and bin gather."""
import os
import socket

import numpy as np
import pytest


def test_chains_for_rank(hq):
    from hubbard_b200.shard import chains_for_rank
    parts = [chains_for_rank(10, r, 3) for r in range(3)]
    assert parts == [[0, 1, 2, 3], [4, 5, 6], [7, 8, 9]]
    assert sum(parts, []) == list(range(10))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime
    import torch.distributed as dist
    from __graft_entry__ import load_package
    hq = load_package()
    from hubbard_b200.shard import chains_for_rank, gather_bins
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = chains_for_rank(5, rank, world)
    bins = {"FillingNumber": np.array([[c + 0.5 * b for b in range(3)] for c in mine]),
            "LocalDensityOfStates": np.array([[[c * 10 + b + t for t in range(4)] for b in range(3)] for c in mine])}
    res = gather_bins(bins, dist)
    if rank == 0:
        np.savez(out_path, **res)
    dist.barrier()
    dist.destroy_process_group()


def test_gather_two_ranks(tmp_path):
    import torch.multiprocessing as tmp
    out = str(tmp_path / "g.npz")
    tmp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    r = np.load(out)
    f = r["FillingNumber"]
    assert f.shape == (5, 3)
    assert np.allclose(f[:, 0], np.arange(5))
    assert r["LocalDensityOfStates"].shape == (5, 3, 4)
    assert r["LocalDensityOfStates"][4, 2, 3] == 4 * 10 + 2 + 3
