"""GPU statistics against the reference's own example run (example/: L=4, u=4, mu=0,
beta=8, nt=160, 1000 warm-up sweeps, all observables), through the measurement schedule
of src/dqmc_handle.cpp with 16 independent chains."""
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_example_run_statistics(hq, golden):
    from hubbard_b200.config import parse_toml_config, chain_params_from
    from hubbard_b200.driver import Handle
    p = parse_toml_config(os.path.join(GOLDEN, "example_config.toml"))
    p.bin_num = 2  # 16 chains x 2 bins = 32 bins (the reference: 20)
    e = hq.Engine(chain_params_from(p, n_chains=16, seed=4242))
    e.fields_random()
    e.init()
    h = Handle(e, p)
    h.thermalize()
    h.measure()
    res = h.analyse(pool_chains=True)
    for key, name in (("filling", "FillingNumber"), ("double_occupancy", "DoubleOccupation"),
                      ("swave", "StaticSWavePairingCorrelation")):
        m, _, err = res[name]
        ref = golden[key]
        assert abs(float(m) - ref["mean"]) < 4 * math.hypot(float(err), ref["stderr"]), (key, m, ref["mean"])
    m, _, err = res["LocalDynamicTransverseSpinCorrelation"]
    ref, rerr = np.array(golden["spin_corr"]["mean"]), np.array(golden["spin_corr"]["stderr"])
    assert np.mean(np.abs(m - ref) < 4 * np.hypot(err, rerr)) > 0.95
    m, _, err = res["LocalDensityOfStates"]
    ref, rerr = np.array(golden["ldos"]["mean"]), np.array(golden["ldos"]["stderr"])
    assert np.mean(np.abs(m - ref) < 4 * np.hypot(err, rerr)) > 0.95
    m, _, err = res["DynamicGreenFunctions"]
    ref = np.array(golden["gf"]["mean"]).reshape(golden["gf"]["nk"], golden["gf"]["nt"])
    rerr = np.array(golden["gf"]["stderr"]).reshape(ref.shape)
    assert np.mean(np.abs(m - ref) < 4 * np.hypot(err, rerr)) > 0.95
    wt, wd = max(e.wrap_errors(c)[0] for c in range(16)), max(e.wrap_errors(c)[1] for c in range(16))
    assert wt < 1e-7 and wd < 1e-7
    e.close()
