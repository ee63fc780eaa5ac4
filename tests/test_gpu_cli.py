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
