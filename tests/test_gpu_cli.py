"""Command-line runs and checkpoints on the GPU: the reference's result files from a short
run, and a resumed run that continues exactly where the checkpointed one stood."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONFIG = """
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
    bin_num = 2
    bin_capacity = 2
    sweeps_between_bins = 2
    observables = ["FillingNumber", "DoubleOccupation", "StaticSWavePairingCorrelation",
                   "DynamicGreenFunctions", "LocalDensityOfStates", "LocalDynamicTransverseSpinCorrelation"]
[Batch]
    chains = 3
    seed = 11
"""


def test_command_line_run_writes_the_reference_files(hq, tmp_path):
    from hubbard_b200 import cli, dqmc_io
    cfg = tmp_path / "config.toml"
    cfg.write_text(CONFIG)
    out = tmp_path / "out"
    assert cli.main(["-c", str(cfg), "-o", str(out), "--checkpoint", str(tmp_path / "ck.npz")]) == 0
    names = {p.name for p in out.iterdir()}
    for stem in ("filling", "double_occu", "swave_corr", "gf", "ldos", "spin_corr"):
        assert stem + ".out" in names and stem + ".bins.out" in names
    assert {"ising.fields", "momenta.out", "tgrids.out"} <= names
    rows = (out / "gf.out").read_text().splitlines()
    assert rows[0].split() == ["9", "10"] and len(rows) == 1 + 9 * 10
    bins = (out / "filling.bins.out").read_text().splitlines()
    assert bins[0].split() == ["6"] and len(bins) == 7  # 3 chains x 2 bins pooled
    fill = [float(x) for x in (out / "filling.out").read_text().splitlines()[1].split()[1:]]
    assert 0.5 < fill[0] < 1.5 and fill[1] >= 0.0 and fill[2] >= 0.0
    f = dqmc_io.load_ising_fields(str(out / "ising.fields"), 10, 16)
    assert set(np.unique(f)) <= {-1, 1}


def test_checkpoint_resume_continues_exactly(hq, tmp_path):
    from hubbard_b200 import dqmc_io
    cfg = [dict(nl=4, u=4.0, beta=2.0, nt=20, stabilization_pace=10, seed=21 + c) for c in range(2)]
    a = hq.Engine(cfg)
    a.fields_random()
    a.init()
    for _ in range(2):
        a.sweep(hq.SWEEP_UP)
        a.sweep(hq.SWEEP_DOWN)
    path = str(tmp_path / "ck.npz")
    dqmc_io.save_checkpoint(path, a, bins={"FillingNumber": np.ones((2, 1))}, meta={"sweeps": 4})
    b = hq.Engine(cfg)
    bins, meta = dqmc_io.load_checkpoint(path, b)
    assert int(meta["sweeps"]) == 4 and bins["FillingNumber"].shape == (2, 1)
    for c in range(2):
        assert np.abs(a.g(c) - b.g(c)).max() <= 1e-12
    for _ in range(2):
        for x in (a, b):
            x.sweep(hq.SWEEP_UP)
            x.sweep(hq.SWEEP_DOWN)
    for c in range(2):
        assert np.array_equal(a.fields(c), b.fields(c))
        assert a.rng_state(c) == b.rng_state(c)
        assert np.abs(a.g(c) - b.g(c)).max() <= 1e-10
    with pytest.raises(hq.HqError):
        b.set_rng_state(0, 0)
    a.close()
    b.close()


def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _cli_rank(rank, world, port, cfg_path, outdir):
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from __graft_entry__ import load_package
    load_package()
    from hubbard_b200 import cli
    # both processes share the one GPU of this test: each runs its own chains on device 0
    assert cli.main(["-c", cfg_path, "-o", outdir, "--device", "0"]) == 0


def test_torchrun_mode_equals_one_process(hq, tmp_path):
    """The command line under torchrun: two processes own chains {0, 1} and {2}, run them
    independently and gather their bins to rank 0, which writes the reference's files. The
    pooled bins equal those of one process running all three chains (chain c keeps seed
    11 + c, whatever the process count)."""
    import torch.multiprocessing as tmp
    from hubbard_b200 import cli
    cfg = tmp_path / "config.toml"
    cfg.write_text(CONFIG)
    one, two = tmp_path / "one", tmp_path / "two"
    assert cli.main(["-c", str(cfg), "-o", str(one)]) == 0
    tmp.start_processes(_cli_rank, args=(2, _free_port(), str(cfg), str(two)), nprocs=2, join=True,
                        start_method="spawn")
    for stem in ("filling", "double_occu", "swave_corr", "gf", "ldos", "spin_corr"):
        a = (one / (stem + ".bins.out")).read_text().splitlines()
        b = (two / (stem + ".bins.out")).read_text().splitlines()
        assert a == b, stem
