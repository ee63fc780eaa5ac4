"""The persistent sweep (one launch per directional sweep) against the launch sequence and the
oracle.

Both modes run the same arithmetic per element of G: every phase of an item of the persistent
kernel (wrap + Metropolis, B chain, UDV, builder GEMMs, inverse) performs the operations of the
kernel it replaces in the same order. So G, the stacks, the fields and the acceptance counts are
compared exactly; only the estimator sums (reduced over 8 instead of 16 warps) are compared at
1e-12 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UP, DOWN = 0, 1


def _metric(n, seed0=1000):
    return [dict(nl=12, u=4.0, mu=0.0, beta=10.0, nt=100, stabilization_pace=10, seed=seed0 + c, expk_mode=-1)
            for c in range(n)]


def _uneven(n, seed0=1000):
    """A mix of the batched uneven configuration: L in {6, 8, 10, 12}, |U| in {2, 4, 6} and beta
    in {4, 8, 12} cycled, dt = 0.1, pace 10."""
    out = []
    for c in range(n):
        beta = [4.0, 8.0, 12.0][(c // 3) % 3]
        out.append(dict(nl=[6, 8, 10, 12][(c * 4) // n], u=[2.0, 4.0, 6.0][c % 3], mu=0.0, beta=beta,
                        nt=int(round(beta / 0.1)), stabilization_pace=10, seed=seed0 + c, expk_mode=-1))
    return out


def _run(hq, params, mode, round_trips, flags=None):
    e = hq.Engine(params)
    e.set_sweep_mode(mode)
    assert e.sweep_mode() == mode
    e.fields_random()
    e.init()
    f = hq.SWEEP_MEASURE if flags is None else flags
    for _ in range(round_trips):
        e.sweep(UP, f)
        e.sweep(DOWN, f)
    e.sync()
    out = dict(G=[e.g(c) for c in range(len(params))], fields=[e.fields(c) for c in range(len(params))],
               est=e.estimators_all(), wrap=[e.wrap_errors(c) for c in range(len(params))],
               stacks=[e.stack(c, 1) for c in range(0, len(params), max(1, len(params) // 4))])
    e.close()
    return out


def _same(a, b):
    for c, (ga, gb) in enumerate(zip(a["G"], b["G"])):
        assert np.array_equal(ga, gb), (c, np.abs(ga - gb).max())
    for c, (fa, fb) in enumerate(zip(a["fields"], b["fields"])):
        assert np.array_equal(fa, fb), c
    # proposals and accepted flips exactly; estimator sums to rounding of their reduction order
    assert np.array_equal(a["est"][:, 4:6], b["est"][:, 4:6])
    np.testing.assert_allclose(a["est"][:, :4], b["est"][:, :4], rtol=1e-12, atol=0)
    assert [w[0] for w in a["wrap"]] == [w[0] for w in b["wrap"]]
    for sa, sb in zip(a["stacks"], b["stacks"]):
        assert sa[0] == sb[0]
        for xa, xb in zip(sa[1:], sb[1:]):
            assert np.array_equal(xa, xb)


def test_persistent_equals_launch_sequence_metric_config(hq):
    """12x12, beta = 10, pace 10: 40 chains (more than fit in one item per SM), two round trips."""
    p = _metric(40)
    _same(_run(hq, p, hq.SWEEP_PERSISTENT, 2), _run(hq, p, hq.SWEEP_LAUNCHES, 2))


def test_persistent_equals_launch_sequence_uneven_chains(hq):
    """Chains of uneven L, U and beta share the queue: 48 chains of the batched uneven mix."""
    p = _uneven(48)
    _same(_run(hq, p, hq.SWEEP_PERSISTENT, 2), _run(hq, p, hq.SWEEP_LAUNCHES, 2))


@pytest.mark.parametrize("k", [4, 8])
def test_persistent_delay_depths(hq, k):
    p = [dict(d, delay_depth=k) for d in _uneven(12)]
    _same(_run(hq, p, hq.SWEEP_PERSISTENT, 1), _run(hq, p, hq.SWEEP_LAUNCHES, 1))


def test_persistent_snapshots_and_dense_expk(hq):
    """Per-slice snapshots (SWEEP_SNAPSHOT) and the dense expK path inside the persistent kernel."""
    p = [dict(nl=6, u=4.0, mu=-0.3, beta=4.0, nt=40, stabilization_pace=10, seed=7 + c, expk_mode=0, snapshots=1)
         for c in range(3)]
    f = hq.SWEEP_MEASURE | hq.SWEEP_SNAPSHOT
    snaps = []
    for mode in (hq.SWEEP_PERSISTENT, hq.SWEEP_LAUNCHES):
        e = hq.Engine(p)
        e.set_sweep_mode(mode)
        e.fields_random()
        e.init()
        e.sweep(UP, f)
        snaps.append([e.g(c, hq.G_TT, t) for c in range(3) for t in range(40)])
        e.close()
    for a, b in zip(*snaps):
        assert np.array_equal(a, b)


def test_persistent_matches_oracle(hq, oracle):
    """4x4, beta = 4 (the CPU-reference configuration) in the persistent mode against the oracle."""
    e = hq.Engine([dict(nl=4, u=4.0, mu=0.0, beta=4.0, nt=40, stabilization_pace=10, seed=42, expk_mode=1)])
    e.set_sweep_mode(hq.SWEEP_PERSISTENT)
    o = oracle.OracleChain(4, u=4.0, mu=0.0, beta=4.0, nt=40, pace=10, seed=42)
    e.fields_random(0)
    o.fields_random()
    e.init()
    o.init()
    for _ in range(2):
        for d in (UP, DOWN):
            e.sweep(d, hq.SWEEP_MEASURE)
            o.sweep(d)
            assert np.array_equal(e.fields(0), o.fields())
            assert np.abs(e.g(0) - o.g()).max() <= 1e-10
    est = e.estimators(0)
    cnt = o.counts()
    assert est[4] == cnt[0] and est[5] == cnt[1]
    e.close()


def test_persistent_is_one_launch_per_sweep(hq):
    """A captured persistent sweep holds one kernel launch (class 'sweep'), whatever the chains."""
    e = hq.Engine(_uneven(16))
    e.set_sweep_mode(hq.SWEEP_PERSISTENT)
    e.fields_random()
    e.init()
    e.profile_enable(True)
    e.capture_graph(UP, hq.SWEEP_MEASURE)
    ms = np.zeros(len(hq.capi.PROFILE_CLASSES))
    cnt = np.zeros(len(hq.capi.PROFILE_CLASSES), dtype=np.int64)
    e.sweep(UP, hq.SWEEP_MEASURE)
    e.profile_collect(ms, cnt)
    i = hq.capi.PROFILE_CLASSES.index("sweep")
    assert cnt[i] == 1 and cnt.sum() == 1 and ms[i] > 0.0
    e.close()


def test_persistent_needs_resident_chains(hq):
    """16 x 16 chains (N = 256) do not fit in one SM: the mode is refused, the context keeps the
    launch sequence."""
    e = hq.Engine([dict(nl=16, u=4.0, mu=-0.2, beta=0.8, nt=16, stabilization_pace=8, seed=5000, expk_mode=-1)])
    with pytest.raises(hq.HqError) as ei:
        e.set_sweep_mode(hq.SWEEP_PERSISTENT)
    assert ei.value.code == hq.capi.HQ_E_RANGE
    assert e.sweep_mode() == hq.SWEEP_LAUNCHES
    e.close()


def test_persistent_phase_cycles(hq):
    """HQ_SWEEP_PHASE_CLOCKS: one item per (chain, interval) counted, every phase timed."""
    p = _uneven(12)
    e = hq.Engine(p)
    e.set_sweep_mode(hq.SWEEP_PERSISTENT)
    e.fields_random()
    e.init()
    e.phase_cycles(reset=True)
    e.sweep(UP, hq.SWEEP_MEASURE | hq.capi.SWEEP_PHASE_CLOCKS)
    pc = e.phase_cycles(reset=True)
    assert pc["items"] == sum(-(-d["nt"] // d["stabilization_pace"]) for d in p)
    for k in ("interval", "bchain", "udt", "push_gemm", "builder_gemm_12", "invert", "builder_gemm_34", "measure"):
        assert pc[k] > 0, k
    e.sweep(DOWN, hq.SWEEP_MEASURE)  # without the flag nothing is counted
    assert e.phase_cycles()["items"] == 0
    e.close()
