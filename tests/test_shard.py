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


def _cli_worker(rank, world, port, outdir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime
    import torch.distributed as dist
    from __graft_entry__ import load_package
    load_package()
    from hubbard_b200.cli import gather_and_write
    from hubbard_b200.config import parse_toml_config
    from hubbard_b200.shard import chains_for_rank
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    p = parse_toml_config(CLI_CONFIG)
    mine = chains_for_rank(5, rank, world)
    nb, nt = p.bin_num, p.nt
    bins = {"FillingNumber": np.array([[1.0 + 0.01 * c + 0.001 * b for b in range(nb)] for c in mine]),
            "LocalDensityOfStates": np.array([[[c + 0.1 * b + 0.01 * t for t in range(nt)] for b in range(nb)]
                                              for c in mine])}
    fields = np.ones((nt, p.nl * p.nl), dtype=np.int32)
    files = gather_and_write(dist, outdir, p, bins, [0], fields)
    assert (files is not None) == (rank == 0)
    dist.barrier()
    dist.destroy_process_group()


CLI_CONFIG = """
[Model.HubbardAttractiveU]
    nnt = 1.0
    u = 4.0
    mu = 0.0
[Lattice.SquareLattice]
    nl = 4
    momentum_list = "AllKstars"
[MonteCarlo]
    beta = 1.0
    nt = 10
    stabilization_pace = 5
    is_fft = false
[Measurement]
    sweeps_warmup = 4
    bin_num = 3
    bin_capacity = 2
    sweeps_between_bins = 2
    observables = ["FillingNumber", "LocalDensityOfStates"]
"""


def test_cli_gather_writes_pooled_bins_on_rank_zero(tmp_path):
    """The command line's torchrun path: two ranks (gloo on CPU) own chains {0,1,2} and {3,4};
    rank 0 writes the result files from the bins of all five chains, in chain order."""
    import torch.multiprocessing as tmp
    out = tmp_path / "out"
    tmp.start_processes(_cli_worker, args=(2, _free_port(), str(out)), nprocs=2, join=True, start_method="spawn")
    rows = (out / "filling.bins.out").read_text().splitlines()
    assert rows[0].split() == ["15"] and len(rows) == 16  # 5 chains x 3 bins pooled
    vals = [float(r.split()[-1]) for r in rows[1:]]
    expect = [1.0 + 0.01 * c + 0.001 * b for c in range(5) for b in range(3)]
    assert np.allclose(vals, expect, rtol=0, atol=1e-12)
    ldos = (out / "ldos.bins.out").read_text().splitlines()
    assert ldos[0].split()[0] == "15"
