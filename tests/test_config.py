"""CPU tests of the configuration mirror (include/dqmc_parser.hpp:49-133)."""
import os

import pytest

from conftest import GOLDEN


def test_example_config(hq):
    from hubbard_b200.config import parse_toml_config, ALL_OBSERVABLES
    p = parse_toml_config(os.path.join(GOLDEN, "example_config.toml"))
    assert (p.nl, p.ns, p.ng, p.nt) == (4, 16, 16, 160)
    assert p.dt == pytest.approx(8.0 / 160)
    assert p.stabilization_pace == 10 and not p.is_fft
    assert p.observable_list == set(ALL_OBSERVABLES)
    assert (p.bin_num, p.bin_capacity, p.sweeps_between_bins, p.sweeps_warmup) == (20, 100, 10, 1000)


def test_bins_divided_by_world_size(hq):
    from hubbard_b200.config import parse_toml_config
    p = parse_toml_config(os.path.join(GOLDEN, "example_config.toml"), world_size=3)
    assert p.bin_num == 7  # ceil(20 / 3)


def test_range_checks_and_observable_options(hq):
    from hubbard_b200.config import parse_toml_config
    base = '[Lattice.SquareLattice]\nmomentum_list = [0, 1]\n[Measurement]\nobservables = ["FillingNumber"]\n'
    with pytest.raises(ValueError, match="'u' out of range"):
        parse_toml_config('[Model.HubbardAttractiveU]\nu = -1.0\n' + base)
    with pytest.raises(ValueError, match="'nt' out of range"):
        parse_toml_config('[MonteCarlo]\nnt = 0\n' + base)
    with pytest.raises(ValueError, match="conflict"):
        parse_toml_config(base.split('[Measurement]')[0] + '[Measurement]\nobservables = ["all", "none"]\n')
    with pytest.raises(ValueError, match="invalid input observables"):
        parse_toml_config(base.split('[Measurement]')[0] + '[Measurement]\nobservables = "all"\n')
    with pytest.raises(ValueError, match="invalid input momentum list"):
        parse_toml_config('[Measurement]\nobservables = ["all"]\n')
    none = parse_toml_config(base.split('[Measurement]')[0] + '[Measurement]\nobservables = ["None"]\n')
    assert none.observable_list == set()


def test_momentum_lists(hq):
    from hubbard_b200.config import momentum_list, kstars
    assert momentum_list(4, "AllKstars") == list(range(9))
    assert momentum_list(4, "X2K2XLine") == [2, 4, 6]
    assert momentum_list(4, "Gamma2MLine") == [0, 4, 8]
    ks = kstars(4)
    assert ks[0] == pytest.approx((0.0, 0.0)) and ks[8] == pytest.approx((3.14159265358979, 3.14159265358979))
    with pytest.raises(ValueError):
        momentum_list(4, [9])


def test_chain_params(hq):
    from hubbard_b200.config import parse_toml_config, chain_params_from
    p = parse_toml_config(os.path.join(GOLDEN, "example_config.toml"))
    cps = chain_params_from(p, n_chains=3, seed=100)
    assert [c["seed"] for c in cps] == [100, 101, 102]
    assert cps[0]["dynamic"] == 1 and cps[0]["nl"] == 4 and cps[0]["nt"] == 160
