"""Measurement schedule, bins and statistics over the C ABI.

Mirrors DQMC::Handle::thermalize / measure / analyse (src/dqmc_handle.cpp:56-168) and the
bin arithmetic of Observable::Observable (include/observable.hpp:168-207), for every
chain of an engine at once. The estimators themselves are accumulated on the GPU inside
the sweep; this module only divides the per-bin sums by the measurement counts and
turns the displacement sums g(d, tau) into G(k, tau).
"""
import math

import numpy as np

from .capi import SWEEP_UP, SWEEP_DOWN, SWEEP_DYNAMIC, SWEEP_MEASURE
from .config import DYNAMIC_OBSERVABLES, EQUALTIME_OBSERVABLES, kstars, momentum_list


def analyse(bins):
    """Mean, population stddev and stderr = stddev / sqrt(nbin) over the bin axis
    (include/observable.hpp:198-207)."""
    bins = np.asarray(bins, dtype=np.float64)
    mean = bins.mean(axis=0)
    std = bins.std(axis=0)
    return mean, std, std / math.sqrt(bins.shape[0])


def gk_from_displacement_sums(gd, nl, klist):
    """G(k, tau) = (1/N) sum_d cos(k . r_d) g(d, tau) (include/observable_methods.hpp:84-103:
    the reference sums exp(-i k (r_j - r_i)) G(j, i); G is real, so only cos contributes).
    gd: [N][nt] displacement sums; returns [nk][nt]."""
    N = nl * nl
    ks = kstars(nl)
    out = np.zeros((len(klist), gd.shape[1]))
    for a, k in enumerate(klist):
        kx, ky = ks[k]
        ph = np.array([math.cos((d % nl) * kx + (d // nl) * ky) for d in range(N)])
        out[a] = ph @ gd / N
    return out


class Handle:
    """Runs the reference's warm-up / measurement schedule on every chain of an engine."""

    def __init__(self, engine, params, use_graphs=True):
        self.e = engine
        self.p = params
        self.use_graphs = use_graphs
        obs = params.observable_list
        self.is_eq = bool(obs & set(EQUALTIME_OBSERVABLES)) and params.bin_num > 0 and params.bin_capacity > 0
        self.is_dyn = bool(obs & set(DYNAMIC_OBSERVABLES)) and params.bin_num > 0 and params.bin_capacity > 0
        self.klist = momentum_list(params.nl, params.momentum_list)
        self.bins = {}

    def _sweep(self, direction, flags=0):
        self.e.sweep(direction, flags)

    def thermalize(self):
        """src/dqmc_handle.cpp:56-87: ceil(w/2) round trips without measurement."""
        for _ in range(int(math.ceil(self.p.sweeps_warmup / 2.0))):
            self._sweep(SWEEP_UP)
            self._sweep(SWEEP_DOWN)
        self.e.sync()

    def measure(self):
        """src/dqmc_handle.cpp:94-162. Returns per-chain bins of every observable."""
        if not (self.is_eq or self.is_dyn):
            return {}
        p, e = self.p, self.e
        n, nt = e.n, p.nt
        binsize = p.bin_capacity if self.is_dyn else int(math.ceil(p.bin_capacity / 2.0))
        eq = np.zeros((n, p.bin_num, 3))
        spin = np.zeros((n, p.bin_num, nt))
        ldos = np.zeros((n, p.bin_num, nt))
        gk = np.zeros((n, p.bin_num, len(self.klist), nt))
        for b in range(p.bin_num):
            for _ in range(int(math.ceil(p.sweeps_between_bins / 2.0))):
                self._sweep(SWEEP_UP)
                self._sweep(SWEEP_DOWN)
            e.reset_estimators(reset_wrap=False)
            n_eq = 0
            for _ in range(binsize):
                if self.is_dyn:
                    self._sweep(SWEEP_DYNAMIC)
                else:
                    self._sweep(SWEEP_UP, SWEEP_MEASURE)
                    n_eq += 1
                self._sweep(SWEEP_DOWN, SWEEP_MEASURE if self.is_eq else 0)
                if self.is_eq:
                    n_eq += 1
            e.sync()
            n_dyn = binsize if self.is_dyn else 0
            for c in range(n):
                est = e.estimators(c)
                if self.is_eq:
                    # per measurement: average over the nt slices of one sweep; per bin: / count
                    eq[c, b] = est[:3] / max(est[3], 1.0)
                if self.is_dyn:
                    sp, ld, gd = e.dynamic_estimators(c)
                    spin[c, b] = sp / n_dyn
                    ldos[c, b] = ld / n_dyn
                    gk[c, b] = gk_from_displacement_sums(gd, p.nl, self.klist) / n_dyn
            _ = n_eq
        out = {}
        if self.is_eq:
            out["FillingNumber"] = eq[:, :, 0]
            out["DoubleOccupation"] = eq[:, :, 1]
            out["StaticSWavePairingCorrelation"] = eq[:, :, 2]
        if self.is_dyn:
            out["LocalDynamicTransverseSpinCorrelation"] = spin
            out["LocalDensityOfStates"] = ldos
            out["DynamicGreenFunctions"] = gk
        self.bins = out
        return out

    def analyse(self, pool_chains=True):
        """Statistics over bins (and over chains as independent bins, the MPI-gather
        analogue of include/utils/observable_gather.hpp:29-79, when pool_chains)."""
        res = {}
        for name, b in self.bins.items():
            data = b.reshape((-1,) + b.shape[2:]) if pool_chains else b[0]
            if name in self.p.observable_list:
                res[name] = analyse(data)
        return res
