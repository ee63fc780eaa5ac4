"""Autotuner (hq_autotune): per lattice size, the expK application (separable circulant
passes or dense DMMA GEMM) and the delay depth are picked by timing whole sweeps, and the
chains continue exactly as if no tuning had run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UP, DOWN = 0, 1


def test_autotune_picks_the_fastest_and_leaves_the_chains_unchanged(hq):
    cfg = [dict(nl=6, u=4.0, beta=4.0, nt=40, stabilization_pace=10, seed=s) for s in (3, 4)]
    cfg.append(dict(nl=4, u=4.0, beta=2.0, nt=20, stabilization_pace=10, seed=5))
    a, b = hq.Engine(cfg), hq.Engine(cfg)
    for x in (a, b):
        x.fields_random()
        x.init()
    table = a.autotune(sweeps=1)
    for nl, chains in ((6, (0, 1)), (4, (2,))):
        rows = [t for t in table if t["nl"] == nl]
        # separable and dense x delay depths 4, 8, 16
        assert len(rows) == 6, rows
        assert sorted({(t["expk_mode"], t["delay_depth"]) for t in rows}) == \
            sorted((m, k) for m in (hq.EXPK_DENSE, hq.EXPK_SEPARABLE) for k in (4, 8, 16))
        assert sum(t["chosen"] for t in rows) == 1
        best = min(rows, key=lambda t: t["ms_per_sweep"])
        assert best["chosen"] and best["ms_per_sweep"] > 0.0
        for c in chains:
            assert a.config(c) == (best["expk_mode"], best["delay_depth"])
    # then the two sweep modes for the whole context (nl = 0); the faster one is in use
    modes = [t for t in table if t["nl"] == 0]
    assert sorted(t["sweep_mode"] for t in modes) == [hq.SWEEP_LAUNCHES, hq.SWEEP_PERSISTENT]
    assert sum(t["chosen"] for t in modes) == 1
    fastest = min(modes, key=lambda t: t["ms_per_sweep"])
    assert fastest["chosen"] and a.sweep_mode() == fastest["sweep_mode"]
    # the tuning sweeps were undone: both engines follow the same trajectory
    for d in (UP, DOWN, UP):
        a.sweep(d, hq.SWEEP_MEASURE)
        b.sweep(d, hq.SWEEP_MEASURE)
    for c in range(3):
        assert np.array_equal(a.fields(c), b.fields(c)), c
        assert np.abs(a.g(c) - b.g(c)).max() <= 1e-10, c
        assert np.abs(a.estimators(c) - b.estimators(c)).max() <= 1e-10 * max(1.0, np.abs(b.estimators(c)).max())
    a.close()
    b.close()


def test_autotune_needs_initialised_stacks(hq):
    e = hq.Engine([dict(nl=4, beta=2.0, nt=20, stabilization_pace=10, seed=1)])
    with pytest.raises(hq.HqError):
        e.autotune(sweeps=1)
    e.fields_random(0)
    e.init()
    with pytest.raises(hq.HqError):
        e.autotune(sweeps=0)
    e.close()


def test_autotune_chooses_the_cluster_size_of_16x16_chains(hq):
    """16 x 16 lattice: the candidates add the interval kernel on four-CTA clusters (separable
    expK, delay depth 16) to the one-CTA ones; the chosen one is the fastest and the chains
    continue exactly as an untuned context (both paths give the same arithmetic)."""
    cfg = [dict(nl=16, u=4.0, mu=-0.2, beta=0.8, nt=16, stabilization_pace=8, seed=5000 + c) for c in range(4)]
    a, b = hq.Engine(cfg), hq.Engine(cfg)
    for x in (a, b):
        x.fields_random()
        x.init()
    table = a.autotune(sweeps=1)
    clustered = [t for t in table if t["cluster_size"] == 4]
    assert len(clustered) == 1 and clustered[0]["expk_mode"] == hq.EXPK_SEPARABLE and clustered[0]["delay_depth"] == 16
    assert len([t for t in table if t["cluster_size"] == 1]) == 6
    # 16 x 16 chains do not fit one SM: no sweep-mode entries, the launch sequence stays
    assert not [t for t in table if t["nl"] == 0] and a.sweep_mode() == hq.SWEEP_LAUNCHES
    assert sum(t["chosen"] for t in table) == 1
    best = min(table, key=lambda t: t["ms_per_sweep"])
    assert best["chosen"]
    for d in (UP, DOWN):
        a.sweep(d, hq.SWEEP_MEASURE)
        b.sweep(d, hq.SWEEP_MEASURE)
    for c in range(4):
        assert np.array_equal(a.fields(c), b.fields(c)), c
        assert np.abs(a.g(c) - b.g(c)).max() <= 1e-10 * max(1.0, np.abs(b.g(c)).max()), c
    a.close()
    b.close()
