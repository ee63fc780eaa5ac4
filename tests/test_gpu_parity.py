"""GPU parity tests: the sm_100a sweep through the C ABI against the CPU oracle.

Tolerances (FP64):
  * G(tau,tau), G(tau,0), G(0,tau): max-abs <= 1e-10 on freshly stabilised slices; on
    wrapped slices each implementation drifts from the exact G by up to its own wrap error
    (the quantity the reference reports), so the bound there is max(1e-10, 2 x (sum of
    both wrap errors)) -- at large beta 10 x the oracle's -- plus a pace-1 comparison
    at 1e-10 relative to max|G|.
  * acceptance ratios of the replayed random stream: 1e-12 relative on the first slice after
    every stabilisation (both G's fresh); median relative 1e-13; max within the G bound of
    wrapped slices times |dr/dG_ii| (~3.5);
  * Ising fields and acceptance counts: identical.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UP, DOWN, DYN = 0, 1, 2


def pair(hq, oracle, L=4, u=4.0, mu=0.0, beta=4.0, nt=40, pace=10, seed=42, mode=1, dynamic=False, snapshots=1,
         delay_depth=0):
    e = hq.Engine([dict(nl=L, u=u, mu=mu, beta=beta, nt=nt, stabilization_pace=pace, seed=seed, expk_mode=mode,
                        dynamic=int(dynamic), snapshots=snapshots, delay_depth=delay_depth)])
    o = oracle.OracleChain(L, u=u, mu=mu, beta=beta, nt=nt, pace=pace, equaltime=True, dynamic=dynamic, seed=seed)
    e.fields_random(0)
    o.fields_random()
    e.init()
    o.init()
    return e, o


@pytest.mark.parametrize("mode", [0, 1], ids=["dense", "separable"])
def test_c1_sweeps_all_slices(hq, oracle, mode):
    """4x4, U=-4, mu=0, beta=4, dt=0.1, pace 10, seed 42 (the CPU-reference config)."""
    e, o = pair(hq, oracle, mode=mode)
    assert np.array_equal(e.fields(0), o.fields())
    assert np.abs(e.g(0) - o.g()).max() <= 1e-10
    for _ in range(2):
        for d in (UP, DOWN):
            e.reset_estimators(reset_wrap=True)
            e.sweep(d, hq.SWEEP_MEASURE | hq.SWEEP_SNAPSHOT)
            o.sweep(d)
            assert np.array_equal(e.fields(0), o.fields())
            errs = np.array([np.abs(e.g(0, hq.G_TT, t) - o.g_slice(0, t)).max() for t in range(40)])
            # freshly stabilised slices (tau = 0, 10, 20, 30): 1e-10 outright
            assert errs[::10].max() <= 1e-10, errs[::10].max()
            # wrapped slices: each implementation drifts from the exact G by up to its wrap
            # error (the reference reports the same quantity); the difference is bounded by both
            floor = max(1e-10, 2.0 * (e.wrap_errors(0)[0] + o.wrap_errors()[0]))
            assert errs.max() <= floor, (errs.max(), floor)
    wt, _ = e.wrap_errors(0)
    assert 0.0 <= wt < 1e-8
    e.close()


def test_c1_acceptance_counts(hq, oracle):
    e, o = pair(hq, oracle)
    for _ in range(2):
        for d in (UP, DOWN):
            e.sweep(d, hq.SWEEP_MEASURE)
            o.sweep(d)
    est = e.estimators(0)
    cnt = o.counts()
    assert est[4] == cnt[0] and est[5] == cnt[1]
    e.close()


def test_ratio_replay(hq, oracle):
    e, o = pair(hq, oracle, seed=7)
    cap = 4 * 40 * 16
    e.ratio_log(0, capacity=cap)
    o.log_ratios(True)
    for d in (UP, DOWN, UP, DOWN):
        e.sweep(d, hq.SWEEP_LOG_RATIOS)
        o.sweep(d)
    rg = e.ratio_log(0)
    ro = o.ratios()
    assert len(rg) == len(ro) == cap
    rel = np.abs(rg - ro) / np.maximum(1.0, np.abs(ro))
    # r = a^2 / (1 + Delta) carries |dr/dG_ii| ~ 3.5 x the G difference; wrapped G's of two
    # implementations differ by up to the sum of their wrap errors (the wrap rounding the
    # reference reports), and right after a stabilisation the ratios agree to ~1e-14
    bound = max(1e-10, 4.0 * 2.0 * (e.wrap_errors(0)[0] + o.wrap_errors()[0]))
    assert rel.max() <= bound, (rel.max(), bound)
    assert np.median(rel) <= 1e-13, np.median(rel)
    # the first slice visited after each stabilisation (steps 0, 10, 20, 30 of every sweep):
    # both G's are freshly built (one wrap away in the up sweep), and the ratios agree to 1e-12
    steps = np.arange(cap) // 16 % 40
    assert rel[steps % 10 == 0].max() <= 1e-12, rel[steps % 10 == 0].max()
    assert np.array_equal(e.fields(0), o.fields())
    e.close()


def test_dynamic_greens_functions(hq, oracle):
    e, o = pair(hq, oracle, dynamic=True)
    for d in (UP, DOWN):
        e.sweep(d)
        o.sweep(d)
    e.sweep(DYN)
    o.sweep(DYN)
    for which, idx in ((hq.G_TT, 0), (hq.G_T0, 1), (hq.G_0T, 2)):
        err = max(np.abs(e.g(0, which, t) - o.g_slice(idx, t)).max() for t in range(40))
        assert err <= 1e-10, (which, err)
    # displaced estimators against the oracle's (include/observable_methods.hpp:110-195)
    sp, ld, gd = e.dynamic_estimators(0)
    osp, old, ogk = o.measure_dynamic(list(range(9)))
    assert np.abs(sp - osp).max() <= 1e-10
    assert np.abs(ld - old).max() <= 1e-10
    from hubbard_b200.driver import gk_from_displacement_sums
    assert np.abs(gk_from_displacement_sums(gd, 4, list(range(9))) - ogk).max() <= 1e-10
    e.close()


@pytest.mark.parametrize("mode", [0, 1], ids=["dense", "separable"])
def test_equaltime_estimators_match_oracle(hq, oracle, mode):
    """Dense mode measures in a pass of its own, separable mode inside the wraps."""
    e, o = pair(hq, oracle, seed=11, mode=mode)
    e.reset_estimators()
    e.sweep(UP, hq.SWEEP_MEASURE)
    o.sweep(UP)
    est = e.estimators(0)
    ref = o.measure_equaltime()
    assert est[3] == 40
    assert np.abs(est[:3] / est[3] - ref).max() <= 1e-10
    # the down sweep measures inside its wraps' last passes, the up sweep in their first
    e.reset_estimators()
    e.sweep(DOWN, hq.SWEEP_MEASURE)
    o.sweep(DOWN)
    est = e.estimators(0)
    ref = o.measure_equaltime()
    assert est[3] == 40
    assert np.abs(est[:3] / est[3] - ref).max() <= 1e-10
    e.close()


def test_c2_single_chain(hq, oracle):
    """8x8, mu=-0.5, beta=8, dt=0.05 (160 slices), pace 10, seed 7, equal-time + displaced G."""
    e, o = pair(hq, oracle, L=8, mu=-0.5, beta=8.0, nt=160, seed=7, dynamic=True)
    for d in (UP, DOWN):
        e.sweep(d, hq.SWEEP_SNAPSHOT)
        o.sweep(d)
        assert np.array_equal(e.fields(0), o.fields())
    e.sweep(DYN)
    o.sweep(DYN)
    floor = max(1e-10, 10 * max(o.wrap_errors()))
    for which, idx in ((hq.G_TT, 0), (hq.G_T0, 1), (hq.G_0T, 2)):
        errs = np.array([np.abs(e.g(0, which, t) - o.g_slice(idx, t)).max() for t in range(160)])
        assert errs.max() <= floor, (which, errs.max(), floor)
        # freshly stabilised slices (every 10th) meet 1e-10 outright
        assert errs[::10].max() <= 1e-10, (which, errs[::10].max())
    e.close()


def test_metric_config_pace_one(hq, oracle):
    """12x12, beta=10, dt=0.1: stabilised every slice, both implementations agree to 1e-10
    relative to the largest entry of G (|G_ij| reaches ~10 in this regime)."""
    e, o = pair(hq, oracle, L=12, beta=10.0, nt=100, pace=1, seed=1000, snapshots=0)
    g = o.g()
    assert np.abs(e.g(0) - g).max() <= 1e-10 * max(1.0, np.abs(g).max())
    e.sweep(UP)
    o.sweep(UP)
    assert np.array_equal(e.fields(0), o.fields())
    g = o.g()
    assert np.abs(e.g(0) - g).max() <= 1e-10 * max(1.0, np.abs(g).max())
    e.close()


def test_metric_config_pace_ten_fields_and_boundary_g(hq, oracle):
    """12x12, beta=10, pace 10 (the benchmark configuration): identical field trajectory,
    G at the stabilisation points within the oracle's own accuracy."""
    e, o = pair(hq, oracle, L=12, beta=10.0, nt=100, pace=10, seed=1000, snapshots=0)
    for d in (UP, DOWN):
        e.sweep(d)
        o.sweep(d)
        assert np.array_equal(e.fields(0), o.fields())
        floor = max(1e-10, 10 * o.wrap_errors()[0])
        assert np.abs(e.g(0) - o.g()).max() <= floor
    e.close()


def test_uneven_batch(hq, oracle):
    """Chains of different L, beta, U in one launch (the batched-chains configuration,
    reduced): each follows its own oracle chain exactly."""
    cfgs = []
    for c in range(6):
        cfgs.append(dict(nl=[4, 6][c % 2], u=[2.0, 4.0, 6.0][c % 3], mu=0.0, beta=[2.0, 4.0][c % 2],
                         nt=[20, 40][c % 2], stabilization_pace=10, seed=1000 + c, expk_mode=-1))
    e = hq.Engine(cfgs)
    orcs = []
    for c, p in enumerate(cfgs):
        e.fields_random(c)
        o = oracle.OracleChain(p["nl"], u=p["u"], beta=p["beta"], nt=p["nt"], pace=10, seed=p["seed"])
        o.fields_random()
        o.init()
        orcs.append(o)
    e.init()
    for d in (UP, DOWN):
        e.sweep(d)
        for o in orcs:
            o.sweep(d)
    for c, o in enumerate(orcs):
        assert np.array_equal(e.fields(c), o.fields()), c
        assert np.abs(e.g(c) - o.g()).max() <= 1e-10, c
    e.close()


def test_uneven_batch_in_chain_groups(hq, oracle):
    """34 chains of uneven L, beta and stack length: enough chains that the initialisation
    and the sweeps run as two chain groups on forked streams. Every chain follows its own
    oracle chain, and the one-copy estimator read equals the per-chain reads."""
    cfgs = []
    for c in range(34):
        cfgs.append(dict(nl=[4, 6][c % 2], u=[2.0, 4.0, 6.0][c % 3], mu=[0.0, -0.3][c % 2],
                         beta=[2.0, 4.0, 3.0][c % 3], nt=[20, 40, 30][c % 3], stabilization_pace=10,
                         seed=2000 + c, expk_mode=-1))
    e = hq.Engine(cfgs)
    orcs = []
    for c, p in enumerate(cfgs):
        e.fields_random(c)
        o = oracle.OracleChain(p["nl"], u=p["u"], mu=p["mu"], beta=p["beta"], nt=p["nt"], pace=10,
                               seed=p["seed"])
        o.fields_random()
        o.init()
        orcs.append(o)
    e.init()
    for c, o in enumerate(orcs):
        assert np.abs(e.g(c) - o.g()).max() <= 1e-10, c
    e.reset_estimators()
    for d in (UP, DOWN):
        e.sweep(d, hq.SWEEP_MEASURE)
        for o in orcs:
            o.sweep(d)
    allest = e.estimators_all()
    assert allest.shape == (34, 6)
    for c, o in enumerate(orcs):
        assert np.array_equal(e.fields(c), o.fields()), c
        assert np.abs(e.g(c) - o.g()).max() <= 1e-10, c
        assert np.array_equal(allest[c], e.estimators(c)), c
        assert allest[c, 3] == 2 * cfgs[c]["nt"], c
    e.close()


def test_graph_replay_is_identical(hq, oracle):
    cfg = dict(nl=6, u=4.0, beta=4.0, nt=40, stabilization_pace=10, seed=5)
    a = hq.Engine([cfg, dict(cfg, seed=6)])
    b = hq.Engine([cfg, dict(cfg, seed=6)])
    for x in (a, b):
        x.fields_random()
        x.init()
    b.capture_graph(UP, hq.SWEEP_MEASURE)
    b.capture_graph(DOWN, hq.SWEEP_MEASURE)
    for d in (UP, DOWN, UP, DOWN):
        a.sweep(d, hq.SWEEP_MEASURE)
        b.sweep(d, hq.SWEEP_MEASURE)
    for c in range(2):
        assert np.array_equal(a.g(c), b.g(c))
        assert np.array_equal(a.fields(c), b.fields(c))
    a.close()
    b.close()


def test_state_errors_are_reported(hq):
    e = hq.Engine([dict(nl=4, beta=2.0, nt=20, stabilization_pace=10, seed=1)])
    with pytest.raises(hq.HqError):
        e.sweep(UP)  # not initialised
    e.fields_random(0)
    e.init()
    with pytest.raises(hq.HqError):
        e.sweep(DOWN)  # stacks at tau = 0
    with pytest.raises(hq.HqError):
        e.set_fields(0, np.full((20, 16), 2))  # fields must be +-1
    with pytest.raises(hq.HqError):
        e.g(0, hq.G_TT, 0)  # no snapshot storage
    e.close()


@pytest.mark.parametrize("delay", [4, 8, 16])
def test_delay_depth_does_not_change_the_chain(hq, oracle, delay):
    e, o = pair(hq, oracle, L=6, seed=3, delay_depth=delay)
    for d in (UP, DOWN):
        e.sweep(d)
        o.sweep(d)
    assert np.array_equal(e.fields(0), o.fields())
    assert np.abs(e.g(0) - o.g()).max() <= 1e-10
    assert e.config(0)[1] == delay
    e.close()


def test_svd_stack_products_match_the_reference(hq, oracle):
    """hq_get_stack (the Utils::SvdStack surface): the product U diag(D) V^T of the top of each
    stack equals the reference's U S V^T of the same B products, at tau = 0 and at beta."""
    e, o = pair(hq, oracle, seed=9)
    for d, side_full in ((None, 1), (UP, 0), (DOWN, 1)):
        if d is not None:
            e.sweep(d)
            o.sweep(d)
        for side in (0, 1):
            n, U, D, V = e.stack(0, side)
            n_ref, prod_ref = o.stack_top(side)
            assert n == n_ref == (4 if side == side_full else 0), (d, side, n, n_ref)
            if n:
                prod = (U * D) @ V.T
                assert np.abs(U.T @ U - np.eye(16)).max() <= 1e-12
                assert np.abs(prod - prod_ref).max() <= 1e-10 * np.abs(prod_ref).max()
    e.close()


def test_c5_lattice_on_the_non_resident_path(hq, oracle):
    """16x16 (N = 256, the C5 lattice): G no longer fits in one SM's shared memory, so every
    kernel runs on its global-memory path. Shortened to beta = 0.8 (16 slices, pace 8)."""
    e, o = pair(hq, oracle, L=16, mu=-0.2, beta=0.8, nt=16, pace=8, seed=5000, snapshots=0)
    assert np.array_equal(e.fields(0), o.fields())
    g = o.g()
    assert np.abs(e.g(0) - g).max() <= 1e-10 * max(1.0, np.abs(g).max())
    for d in (UP, DOWN):
        e.sweep(d, hq.SWEEP_MEASURE)
        o.sweep(d)
        assert np.array_equal(e.fields(0), o.fields())
        g = o.g()
        floor = max(1e-10, 10 * o.wrap_errors()[0])
        assert np.abs(e.g(0) - g).max() <= floor * max(1.0, np.abs(g).max())
    est = e.estimators(0)
    assert est[4] == 2 * 16 * 256 and est[5] == o.counts()[1]
    e.close()


def test_profiling_with_and_without_graphs(hq):
    """Per-launch device times (hq_profile_collect) of a plain sweep and of a graph replay, in
    the launch-sequence mode (one interval launch per stabilisation interval)."""
    e = hq.Engine([dict(nl=4, u=4.0, beta=4.0, nt=40, stabilization_pace=10, seed=2)])
    e.set_sweep_mode(hq.SWEEP_LAUNCHES)
    e.fields_random()
    e.init()
    e.profile_enable(True)
    classes = hq.capi.PROFILE_CLASSES
    for use_graph, d in ((False, UP), (True, DOWN)):
        if use_graph:
            e.capture_graph(d, hq.SWEEP_MEASURE)
        ms = np.zeros(len(classes))
        cnt = np.zeros(len(classes), dtype=np.int64)
        e.sweep(d, hq.SWEEP_MEASURE)
        e.profile_collect(ms, cnt)
        i = classes.index("interval")
        assert cnt[i] == 4 and ms[i] > 0.0, (use_graph, cnt, ms)
    e.close()


def test_c5_cluster_path_equals_global_memory_path(hq, oracle):
    """16x16: the interval kernel on four-CTA clusters (G in the cluster's distributed shared
    memory) against the one-CTA kernel with G in global memory (HQ_INTERVAL_CLUSTER=0): the
    same fields, counts and G (each element sees the same floating-point operations), and the
    oracle's fields. 8 chains, beta = 1.6 (32 slices, pace 8), snapshots and ratio log on."""
    import os
    cfgs = [dict(nl=16, u=4.0, mu=-0.2, beta=1.6, nt=32, stabilization_pace=8, seed=5000 + c, expk_mode=1,
                 snapshots=1) for c in range(8)]
    engines = []
    for cluster in (True, False):
        if not cluster:
            os.environ["HQ_INTERVAL_CLUSTER"] = "0"
        try:
            e = hq.Engine(cfgs)
        finally:
            os.environ.pop("HQ_INTERVAL_CLUSTER", None)
        e.fields_random()
        e.init()
        e.ratio_log(0, capacity=4 * 32 * 256)
        e.profile_enable(True)
        engines.append(e)
    classes = hq.capi.PROFILE_CLASSES
    o = oracle.OracleChain(16, u=4.0, mu=-0.2, beta=1.6, nt=32, pace=8, seed=5000)
    o.fields_random()
    o.init()
    a, b = engines
    for d in (UP, DOWN, UP, DOWN):
        counts = []
        for e in engines:
            ms = np.zeros(len(classes))
            cnt = np.zeros(len(classes), dtype=np.int64)
            e.sweep(d, hq.SWEEP_MEASURE | hq.SWEEP_SNAPSHOT | hq.SWEEP_LOG_RATIOS)
            e.profile_collect(ms, cnt)
            counts.append(cnt)
        o.sweep(d)
        assert counts[0][classes.index("interval_cluster")] == 4 and counts[0][classes.index("interval")] == 0
        assert counts[1][classes.index("interval")] == 4 and counts[1][classes.index("interval_cluster")] == 0
        assert np.array_equal(a.fields(0), o.fields())
        for c in range(8):
            assert np.array_equal(a.fields(c), b.fields(c)), c
            assert np.abs(a.g(c) - b.g(c)).max() <= 1e-13, (c, np.abs(a.g(c) - b.g(c)).max())
            for t in range(0, 32, 5):
                assert np.abs(a.g(c, hq.G_TT, t) - b.g(c, hq.G_TT, t)).max() <= 1e-13, (c, t)
        ea, eb = a.estimators_all(), b.estimators_all()
        assert np.array_equal(ea[:, 3:], eb[:, 3:])
        assert np.abs(ea[:, :3] - eb[:, :3]).max() <= 1e-12 * np.abs(eb[:, :3]).max()
    assert np.array_equal(a.ratio_log(0), b.ratio_log(0))
    g = o.g()
    assert np.abs(a.g(0) - g).max() <= 1e-10 * max(1.0, np.abs(g).max())
    for e in engines:
        e.close()
