"""CPU tests of the oracle (the checker of the CUDA path).

The reference cannot be compiled in this image (Eigen, MKL, Boost, xtensor are absent),
so the oracle is pinned against the reference's own example run: its final Ising field
configuration, its wrap-error scale and its binned observables (tests/golden/)."""
import math
import random

import numpy as np
import pytest

from conftest import example_fields


def test_rng_is_libstdcxx_minstd_rand0(oracle):
    # std::default_random_engine == minstd_rand0: x <- 16807 x mod (2^31 - 1), seeded by set_seed
    c = oracle.OracleChain(4, seed=42)
    draws = c.engine_draws(5)
    x = 42
    ref = []
    for _ in range(5):
        x = (16807 * x) % 2147483647
        ref.append(x)
    assert list(draws) == ref


def test_canonical_uses_two_draws(oracle):
    # generate_canonical<double,53> on a 31-bit engine consumes two values per variate
    a = oracle.OracleChain(4, seed=7)
    b = oracle.OracleChain(4, seed=7)
    u = a.canonical_draws(3)
    raw = b.engine_draws(6).astype(np.float64)
    R = 2147483646.0
    for k in range(3):
        s = (raw[2 * k] - 1.0) + (raw[2 * k + 1] - 1.0) * R
        assert u[k] == s / (R * R)


def test_fields_from_seed_follow_bernoulli_half(oracle):
    c = oracle.OracleChain(4, beta=4.0, nt=40, seed=42)
    c.fields_random()
    f = c.fields()
    d = oracle.OracleChain(4, beta=4.0, nt=40, seed=42)
    u = d.canonical_draws(40 * 16).reshape(40, 16)
    assert np.array_equal(f, np.where(u < 0.5, 1, -1))


def test_expk_matches_dense_exponential(oracle):
    c = oracle.OracleChain(4, mu=-0.5, beta=4.0, nt=40)
    E, Ei = c.expk()
    # K = -t H_nn - mu; exp(-dt K) exp(+dt K) = 1 and E symmetric
    assert np.abs(E @ Ei - np.eye(16)).max() < 1e-13
    assert np.abs(E - E.T).max() < 1e-15


def test_example_fields_wrap_error_scale(oracle, golden):
    # the reference's final field configuration of example/ with example/config.toml:
    # the wrap error of a no-update pass is of the scale the reference reports (log.out)
    f = example_fields()
    c = oracle.OracleChain(4, u=4.0, mu=0.0, beta=8.0, nt=160, pace=10, equaltime=True, dynamic=True, seed=1)
    c.set_fields(f)
    c.init()
    c.sweep(oracle.DYNAMIC)
    tt, dyn = c.wrap_errors()
    assert 0 <= tt < 100 * golden["wrap_error"]["equaltime"]
    assert 0 <= dyn < 100 * max(golden["wrap_error"]["dynamic"], 1e-12)


def test_g_of_example_fields_is_exact_inverse(oracle):
    # G(0,0) = (1 + B(nt-1)...B(0))^-1 for the example field configuration, checked against a
    # direct long-double-free evaluation at small beta where the product is well conditioned
    f = example_fields()[:40]
    c = oracle.OracleChain(4, u=4.0, beta=2.0, nt=40, pace=10, seed=1)
    c.set_fields(f)
    c.init()
    E, _ = c.expk()
    a = c.alpha
    X = np.eye(16)
    for t in range(1, 41):
        X = (np.exp(a * f[t % 40])[:, None] * E) @ X
    # initial G is G(beta, beta) = (1 + B(0) B(39) ... B(1))^-1
    Y = np.eye(16)
    for t in range(1, 41):
        Y = (np.exp(a * f[t % 40])[:, None] * E) @ Y
    G = np.linalg.inv(np.eye(16) + Y)
    assert np.abs(c.g() - G).max() < 1e-10  # the unstabilised direct product limits this check


def test_sweep_keeps_g_consistent_with_stacks(oracle):
    c = oracle.OracleChain(4, beta=4.0, nt=40, pace=10, seed=42)
    c.fields_random()
    c.init()
    for _ in range(3):
        c.sweep(oracle.UP)
        c.sweep(oracle.DOWN)
    tt, _ = c.wrap_errors()
    assert tt < 1e-9
    n_prop, n_acc = c.counts()
    assert n_prop == 6 * 40 * 16 and 0 < n_acc < n_prop


def test_estimator_definitions(oracle):
    c = oracle.OracleChain(4, beta=4.0, nt=40, pace=10, seed=3, equaltime=True)
    c.fields_random()
    c.init()
    c.sweep(oracle.UP)
    f, dd, sw = c.measure_equaltime()
    Gs = [c.g_slice(0, t) for t in range(40)]
    N = 16
    assert abs(f - np.mean([2 - 2 * np.trace(g) / N for g in Gs])) < 1e-12
    assert abs(dd - np.mean([np.sum((1 - np.diag(g)) ** 2) / N for g in Gs])) < 1e-12
    ref = np.mean([np.sum((np.eye(N) - g).T ** 2 + g ** 2) / N for g in Gs])
    assert abs(sw - ref) < 1e-12


def test_analyse_population_stddev():
    from oracle.oracle import analyse
    x = np.array([1.0, 2.0, 4.0])
    m, s, e = analyse(x)
    assert m == pytest.approx(7 / 3)
    assert s == pytest.approx(np.sqrt(np.mean((x - 7 / 3) ** 2)))
    assert e == pytest.approx(s / math.sqrt(3))


@pytest.mark.slow
def test_oracle_reproduces_example_observables(oracle, golden):
    """The reference's own run (example/: L=4, u=4, mu=0, beta=8, nt=160, 1000 warm-up,
    20 bins x 100, all observables) reproduced by the oracle within combined error bars."""
    c = oracle.OracleChain(4, u=4.0, mu=0.0, beta=8.0, nt=160, pace=10, equaltime=True, dynamic=True, seed=2024)
    c.fields_random()
    c.init()
    r = c.run_schedule(1000, 20, 100, 10, equaltime=True, dynamic=True, klist=list(range(9)))
    for k, key in enumerate(["filling", "double_occupancy", "swave"]):
        m, _, e = oracle.analyse(r["eq"][:, k])
        ref = golden[key]
        assert abs(m - ref["mean"]) < 4 * math.hypot(e, ref["stderr"]), (key, m, ref["mean"])
    ms, _, es = oracle.analyse(r["spin"])
    ref = np.array(golden["spin_corr"]["mean"])
    refe = np.array(golden["spin_corr"]["stderr"])
    z = np.abs(ms - ref) / np.hypot(es, refe)
    assert np.mean(z < 4) > 0.95
