"""The batched, single-chain, adjoint and large configurations at their stated sizes.

  C2  8x8, mu=-0.5, beta=8, dt=0.05 (nt=160), pace 10, seed 7: 200 warm-up + 500 measurement
      sweeps in 20 bins (each an updating sweep paired with a no-update dynamic pass,
      src/dqmc_handle.cpp:131-142); binned filling, double occupancy, s-wave and spin
      correlation against the oracle running the same schedule and seed.
  C3  256 chains, L in {6,8,10,12} (64 each), |U| in {2,4,6} and beta in {4,8,12} cycled
      (dt=0.1, nt in {40,80,120}), pace 10, seeds 1000+c, delay depth autotuned; after two
      round trips one chain of each (L, U, beta) class against its oracle chain.
  C4  10x10, mu=-0.3, |U|=4, beta=6, nt=60, 64 configurations from seed 99: dmu, dalpha and
      four bond hoppings of 8 configurations against central differences (h=1e-5).
  C5  64 chains of 16x16 (N=256), mu=-0.2, beta=16, dt=0.05 (nt=320), pace 8, seeds 5000+c:
      one round trip of all chains, chains 0 and 63 against the oracle.

Tolerances: identical field trajectories; G after each sweep within 5e-9 x max|G| of the
pace-10 oracle (the oracle's own SVD-stack accuracy at large beta; 1e-10 where beta is
small, as in tests/test_gpu_parity.py); binned statistics equal to 1e-9 when the
trajectories coincide and within 3 combined standard errors in any case; gradients within
1e-6 relative of the central differences.
"""
import math
import multiprocessing as mp

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

UP, DOWN, DYN = 0, 1, 2


# ------------------------------------------------------------------------------------
#  C2: the full measurement schedule
# ------------------------------------------------------------------------------------
C2 = dict(nl=8, nnt=1.0, u=4.0, mu=-0.5, beta=8.0, nt=160, stabilization_pace=10)
C2_SCHEDULE = dict(sweeps_warmup=200, bin_num=20, bin_capacity=25, sweeps_between_bins=0)


def _c2_oracle(seed):
    from oracle.oracle import OracleChain, set_num_threads
    set_num_threads(1)
    o = OracleChain(C2["nl"], nnt=C2["nnt"], u=C2["u"], mu=C2["mu"], beta=C2["beta"], nt=C2["nt"],
                    pace=C2["stabilization_pace"], equaltime=True, dynamic=True, seed=seed)
    o.fields_random()
    o.init()
    res = o.run_schedule(C2_SCHEDULE["sweeps_warmup"], C2_SCHEDULE["bin_num"], C2_SCHEDULE["bin_capacity"],
                         C2_SCHEDULE["sweeps_between_bins"], equaltime=True, dynamic=True)
    res["fields"] = o.fields()
    return res


def test_c2_measurement_schedule(hq):
    from hubbard_b200.config import Params
    from hubbard_b200.driver import Handle, analyse
    seed = 7
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        job = pool.apply_async(_c2_oracle, (seed,))
        p = Params()
        p.nl, p.nnt, p.u, p.mu, p.beta, p.nt = C2["nl"], C2["nnt"], C2["u"], C2["mu"], C2["beta"], C2["nt"]
        p.stabilization_pace = C2["stabilization_pace"]
        for k, v in C2_SCHEDULE.items():
            setattr(p, k, v)
        p.observable_list = {"FillingNumber", "DoubleOccupation", "StaticSWavePairingCorrelation",
                             "LocalDynamicTransverseSpinCorrelation"}
        e = hq.Engine([dict(C2, seed=seed, expk_mode=-1, dynamic=1)])
        e.fields_random()
        e.init()
        h = Handle(e, p)
        h.thermalize()
        bins = h.measure()
        gpu_fields = e.fields(0)
        wrap = e.wrap_errors(0)
        e.close()
        ref = job.get(timeout=1200)
    assert bins["FillingNumber"].shape == (1, 20)
    same = np.array_equal(gpu_fields, ref["fields"])
    pairs = [("FillingNumber", ref["eq"][:, 0]), ("DoubleOccupation", ref["eq"][:, 1]),
             ("StaticSWavePairingCorrelation", ref["eq"][:, 2]),
             ("LocalDynamicTransverseSpinCorrelation", ref["spin"])]
    for name, rb in pairs:
        gb = bins[name][0]
        gm, _, ge = analyse(gb)
        rm, _, re_ = analyse(rb)
        if same:
            assert np.abs(gb - rb).max() <= 1e-9, (name, np.abs(gb - rb).max())
        z = np.abs(gm - rm) / np.maximum(np.hypot(ge, re_), 1e-300)
        assert np.all(z <= 3.0), (name, z.max())
    assert same, "field trajectories of the C2 schedule diverged"
    assert wrap[0] < 1e-7 and wrap[1] < 1e-7


# ------------------------------------------------------------------------------------
#  C3: 256 chains of uneven L, U and beta
# ------------------------------------------------------------------------------------
def c3_chains():
    out = []
    for c in range(256):
        beta = [4.0, 8.0, 12.0][(c // 3) % 3]
        out.append(dict(nl=[6, 8, 10, 12][c // 64], nnt=1.0, u=[2.0, 4.0, 6.0][c % 3], mu=0.0, beta=beta,
                        nt=int(round(beta / 0.1)), stabilization_pace=10, seed=1000 + c, expk_mode=-1))
    return out


def _c3_oracle(args):
    cfg, sweeps = args
    from oracle.oracle import OracleChain, set_num_threads
    set_num_threads(1)
    o = OracleChain(cfg["nl"], nnt=cfg["nnt"], u=cfg["u"], mu=cfg["mu"], beta=cfg["beta"], nt=cfg["nt"],
                    pace=cfg["stabilization_pace"], seed=cfg["seed"])
    o.fields_random()
    o.init()
    for k in range(sweeps):
        o.sweep(k % 2)
    return o.fields(), o.g(), o.counts()


def test_c3_batched_uneven_chains(hq):
    cfgs = c3_chains()
    classes = {}
    for c, p in enumerate(cfgs):
        classes.setdefault((p["nl"], p["u"], p["beta"]), c)
    reps = sorted(classes.values())
    assert len(reps) == 36
    ctx = mp.get_context("spawn")
    with ctx.Pool(8) as pool:
        job = pool.map_async(_c3_oracle, [(cfgs[c], 4) for c in reps])
        e = hq.Engine(cfgs)
        e.fields_random()
        e.init()
        tune = e.autotune(sweeps=1)
        assert any(t["chosen"] for t in tune)
        for k in range(4):
            e.sweep(k % 2, hq.SWEEP_MEASURE)
        est = e.estimators_all()
        got = [(e.fields(c), e.g(c)) for c in reps]
        e.close()
        ref = job.get(timeout=1200)
    for (c, (gf, gg), (rf, rg, rc)) in zip(reps, got, ref):
        assert np.array_equal(gf, rf), cfgs[c]
        assert np.abs(gg - rg).max() <= 5e-9 * max(1.0, np.abs(rg).max()), (cfgs[c], np.abs(gg - rg).max())
        assert est[c, 4] == rc[0] and est[c, 5] == rc[1], cfgs[c]
    # every chain measured all its slices: 4 sweeps x nt
    assert np.array_equal(est[:, 3], np.array([4.0 * p["nt"] for p in cfgs]))


# ------------------------------------------------------------------------------------
#  C4: finite differences of the log-det adjoint on 8 of the 64 configurations
# ------------------------------------------------------------------------------------
def _nn_hop(L):
    N = L * L
    H = np.zeros((N, N))
    for s in range(N):
        x, y = s % L, s // L
        for t in ((x + 1) % L + L * y, x + L * ((y + 1) % L)):
            H[s, t] += 1.0
            H[t, s] += 1.0
    return H


C4 = dict(L=10, beta=6.0, nt=60, mu=-0.3, u=4.0)
C4_PICK = (0, 9, 18, 27, 36, 45, 54, 63)
C4_BONDS = ((0, 1), (0, 10), (44, 45), (99, 9))


def _c4_fd(args):
    c, fields = args
    from oracle.oracle import OracleChain, set_num_threads
    set_num_threads(1)
    L, beta, nt, mu, u = C4["L"], C4["beta"], C4["nt"], C4["mu"], C4["u"]
    hop = _nn_hop(L)
    h = 1e-5

    def logdet(mu_=mu, u_=u, hop_=hop):
        q = OracleChain(L, u=u_, mu=mu_, beta=beta, nt=nt, pace=10, seed=1, custom_hop=hop_)
        q.set_fields(fields)
        return q.logdet()

    out = {"mu": (logdet(mu_=mu + h) - logdet(mu_=mu - h)) / (2 * h),
           "u": (logdet(u_=u + h) - logdet(u_=u - h)) / (2 * h), "bonds": []}
    for (i, j) in C4_BONDS:
        hp, hm = hop.copy(), hop.copy()
        hp[i, j] += h
        hp[j, i] += h
        hm[i, j] -= h
        hm[j, i] -= h
        out["bonds"].append((logdet(hop_=hp) - logdet(hop_=hm)) / (2 * h))
    return out


def test_c4_finite_differences_of_eight_configurations(hq, oracle):
    L, beta, nt, mu, u = C4["L"], C4["beta"], C4["nt"], C4["mu"], C4["u"]
    hop = _nn_hop(L)
    for (i, j) in C4_BONDS:
        assert hop[i, j] == 1.0
    src = oracle.OracleChain(L, nt=nt, beta=1.0, seed=99)
    fields = []
    for _ in range(64):
        src.fields_random()
        fields.append(src.fields())
    ctx = mp.get_context("spawn")
    with ctx.Pool(8) as pool:
        job = pool.map_async(_c4_fd, [(c, fields[c]) for c in C4_PICK])
        e = hq.Engine([dict(nl=L, u=u, mu=mu, beta=beta, nt=nt, stabilization_pace=10, seed=c, expk_mode=0)
                       for c in range(64)])
        for c in range(64):
            e.set_hopping(c, hop)
            e.set_fields(c, fields[c])
        e.init()
        _, grads = e.logdet_adjoint()
        e.close()
        fd = job.get(timeout=1200)
    dt = beta / nt
    dalpha_du = 0.5 * dt * math.exp(0.5 * dt * u) / math.sqrt(math.exp(dt * u) - 1.0)
    for c, f in zip(C4_PICK, fd):
        g_mu, g_al, g_K = grads[c]
        assert abs(g_mu - f["mu"]) <= 1e-6 * max(1.0, abs(f["mu"])), (c, g_mu, f["mu"])
        assert abs(g_al * dalpha_du - f["u"]) <= 1e-6 * max(1.0, abs(f["u"])), (c, g_al * dalpha_du, f["u"])
        for (i, j), fb in zip(C4_BONDS, f["bonds"]):
            g_b = -(g_K[i, j] + g_K[j, i])
            assert abs(g_b - fb) <= 1e-6 * max(1.0, abs(fb)), (c, i, j, g_b, fb)


# ------------------------------------------------------------------------------------
#  C5: 64 chains of 16 x 16 at beta = 16
# ------------------------------------------------------------------------------------
C5 = dict(nl=16, nnt=1.0, u=4.0, mu=-0.2, beta=16.0, nt=320, stabilization_pace=8)


def _c5_oracle(seed):
    from oracle.oracle import OracleChain, set_num_threads
    set_num_threads(1)
    o = OracleChain(C5["nl"], nnt=C5["nnt"], u=C5["u"], mu=C5["mu"], beta=C5["beta"], nt=C5["nt"],
                    pace=C5["stabilization_pace"], seed=seed)
    o.fields_random()
    o.init()
    out = []
    for d in (UP, DOWN):
        o.sweep(d)
        out.append((o.fields(), o.g()))
    return out, o.counts()


def test_c5_full_size(hq):
    picks = (0, 63)
    ctx = mp.get_context("spawn")
    with ctx.Pool(2) as pool:
        job = pool.map_async(_c5_oracle, [5000 + c for c in picks])
        e = hq.Engine([dict(C5, seed=5000 + c, expk_mode=-1) for c in range(64)])
        e.fields_random()
        e.init()
        got = []
        for d in (UP, DOWN):
            e.sweep(d, hq.SWEEP_MEASURE)
            got.append([(e.fields(c), e.g(c)) for c in picks])
        est = e.estimators_all()
        e.close()
        ref = job.get(timeout=1200)
    for k, c in enumerate(picks):
        sweeps, counts = ref[k]
        for d in range(2):
            gf, gg = got[d][k]
            rf, rg = sweeps[d]
            assert np.array_equal(gf, rf), (c, d)
            assert np.abs(gg - rg).max() <= 5e-9 * max(1.0, np.abs(rg).max()), (c, d, np.abs(gg - rg).max())
        assert est[c, 4] == counts[0] and est[c, 5] == counts[1]
    assert np.all(est[:, 3] == 2 * C5["nt"])
