"""CPU tests of the measurement schedule (src/dqmc_handle.cpp:56-162) with a recording
fake engine, and of the G(k, tau) transform."""
import math

import numpy as np
import pytest


class FakeEngine:
    def __init__(self, n, nt, N):
        self.n, self.nt, self.N = n, nt, N
        self.calls = []
        self.acc = np.zeros((n, 6))

    def sweep(self, d, flags=0):
        self.calls.append((d, flags))
        if flags & 1:
            self.acc[:, :4] += [1.0 * self.nt, 0.5 * self.nt, 2.0 * self.nt, self.nt]

    def sync(self):
        pass

    def reset_estimators(self, reset_wrap=False):
        self.acc[:] = 0.0

    def estimators(self, c):
        return self.acc[c].copy()

    def dynamic_estimators(self, c):
        return np.ones(self.nt), np.ones(self.nt), np.ones((self.N, self.nt))


def make(hq, obs, **kw):
    from hubbard_b200.config import parse_toml_config
    o = ", ".join('"%s"' % x for x in obs)
    txt = ("[Lattice.SquareLattice]\nnl = 4\nmomentum_list = \"AllKstars\"\n[MonteCarlo]\nnt = 8\n[Measurement]\nsweeps_warmup = %d\nbin_num = %d\n"
           "bin_capacity = %d\nsweeps_between_bins = %d\nobservables = [%s]\n"
           % (kw.get("w", 5), kw.get("bins", 2), kw.get("cap", 3), kw.get("between", 3), o))
    return parse_toml_config(txt)


def test_schedule_equaltime(hq):
    from hubbard_b200.driver import Handle
    p = make(hq, ["FillingNumber"])
    e = FakeEngine(2, 8, 16)
    h = Handle(e, p)
    h.thermalize()
    assert len(e.calls) == 2 * math.ceil(5 / 2)
    e.calls.clear()
    bins = h.measure()
    # per bin: ceil(3/2) round trips between bins + ceil(3/2) measuring round trips
    assert len(e.calls) == 2 * (2 * 2 + 2 * 2)
    assert bins["FillingNumber"].shape == (2, 2)
    assert np.allclose(bins["FillingNumber"], 1.0)
    assert np.allclose(bins["StaticSWavePairingCorrelation"], 2.0)


def test_schedule_dynamic(hq):
    from hubbard_b200.driver import Handle
    from hubbard_b200.capi import SWEEP_DYNAMIC, SWEEP_DOWN
    p = make(hq, ["LocalDensityOfStates", "FillingNumber"], cap=4)
    e = FakeEngine(1, 8, 16)
    h = Handle(e, p)
    bins = h.measure()
    dyn = [c for c in e.calls if c[0] == SWEEP_DYNAMIC]
    assert len(dyn) == 2 * 4  # bin_capacity dynamic passes per bin
    assert all(f == 1 for d, f in e.calls if d == SWEEP_DOWN and (d, f) in e.calls[-8:])
    assert np.allclose(bins["LocalDensityOfStates"], 1.0 / 4)


def test_gk_transform(hq):
    from hubbard_b200.driver import gk_from_displacement_sums
    nl, nt = 4, 3
    N = nl * nl
    rng = np.random.default_rng(0)
    G = rng.normal(size=(N, N))
    # brute force of include/observable_methods.hpp:84-103 with the displacement table
    from hubbard_b200.config import kstars
    ks = kstars(nl)
    gd = np.zeros((N, nt))
    for d in range(N):
        dx, dy = d % nl, d // nl
        for i in range(N):
            xi, yi = i % nl, i // nl
            j = (xi + dx) % nl + nl * ((yi + dy) % nl)
            gd[d, :] += G[j, i]
    out = gk_from_displacement_sums(gd, nl, list(range(9)))
    for k, (kx, ky) in enumerate(ks):
        ref = 0.0
        for i in range(N):
            for j in range(N):
                rx = ((j % nl) - (i % nl) + nl) % nl
                ry = ((j // nl) - (i // nl) + nl) % nl
                ref += (np.exp(-1j * (kx * rx + ky * ry)) * G[j, i]).real / N
        assert out[k, 0] == pytest.approx(ref, abs=1e-12)


def test_analyse(hq):
    from hubbard_b200.driver import analyse
    m, s, e = analyse(np.array([[1.0], [3.0]]))
    assert m[0] == 2.0 and s[0] == 1.0 and e[0] == pytest.approx(1 / math.sqrt(2))
