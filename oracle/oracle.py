"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference DQMC sweep on the CPU (see dqmc_oracle.cpp for the
function-by-function citations). Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline legs import this module, as the checker -- the product never does.
"""
import ctypes
import math
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.OUT
        if not os.path.exists(path):
            _build.build()
        L = ctypes.CDLL(path)
        vp, i, d, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
        dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.or_create.restype = vp
        L.or_create.argtypes = [i, d, d, d, d, i, i, i, i, ll, dp]
        L.or_destroy.argtypes = [vp]
        L.or_alpha.restype = d
        L.or_alpha.argtypes = [vp]
        L.or_get_expk.argtypes = [vp, dp, dp]
        L.or_fields_random.argtypes = [vp]
        L.or_set_fields.argtypes = [vp, ip]
        L.or_get_fields.argtypes = [vp, ip]
        L.or_engine_draws.argtypes = [vp, ll, ctypes.POINTER(ctypes.c_uint)]
        L.or_canonical_draws.argtypes = [vp, ll, dp]
        L.or_init.restype = i
        L.or_init.argtypes = [vp]
        L.or_set_thermalization.argtypes = [vp, i]
        L.or_set_forced_fields.argtypes = [vp, ip]
        L.or_sweep.restype = i
        L.or_sweep.argtypes = [vp, i]
        L.or_current_g.argtypes = [vp, dp]
        L.or_get_g.restype = i
        L.or_get_g.argtypes = [vp, i, i, dp]
        L.or_current_dyn.argtypes = [vp, dp, dp]
        L.or_wrap_errors.argtypes = [vp, dp]
        L.or_counts.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.or_set_ratio_log.argtypes = [vp, i]
        L.or_ratio_log.restype = ll
        L.or_ratio_log.argtypes = [vp, dp, ll]
        L.or_measure_equaltime.argtypes = [vp, dp]
        L.or_measure_dynamic.argtypes = [vp, dp, dp, ip, i, dp]
        L.or_nkstars.restype = i
        L.or_nkstars.argtypes = [vp]
        L.or_run_schedule.restype = i
        L.or_run_schedule.argtypes = [vp, i, i, i, i, i, i, ip, i, dp, dp, dp, dp]
        L.or_logdet.restype = d
        L.or_stack_top.restype = i
        L.or_stack_top.argtypes = [vp, i, dp]
        L.or_logdet.argtypes = [vp]
        L.or_logdet_grad.restype = i
        L.or_logdet_grad.argtypes = [vp, dp]
        L.or_set_num_threads.argtypes = [i]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


UP, DOWN, DYNAMIC = 0, 1, 2


class OracleChain:
    """One Markov chain of the CPU restatement (model + core + its own engine)."""

    def __init__(self, nl, nnt=1.0, u=4.0, mu=0.0, beta=8.0, nt=160, pace=10, equaltime=True, dynamic=False,
                 seed=0, custom_hop=None):
        self.nl, self.ns, self.nt, self.pace = nl, nl * nl, nt, pace
        self.nnt, self.u, self.mu, self.beta = nnt, u, mu, beta
        self.dt = beta / nt
        hop = None
        if custom_hop is not None:
            self._hop = np.asfortranarray(custom_hop, dtype=np.float64)
            hop = _dp(self._hop)
        self.h = lib().or_create(nl, nnt, u, mu, beta, nt, pace, int(equaltime), int(dynamic), int(seed), hop)
        if not self.h:
            raise RuntimeError("or_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_destroy(self.h)
            self.h = None

    @property
    def alpha(self):
        return lib().or_alpha(self.h)

    def expk(self):
        a = np.zeros((self.ns, self.ns), order="F")
        b = np.zeros((self.ns, self.ns), order="F")
        lib().or_get_expk(self.h, _dp(a), _dp(b))
        return a, b

    def fields_random(self):
        lib().or_fields_random(self.h)

    def set_fields(self, f):
        f = np.ascontiguousarray(f, dtype=np.int32).reshape(self.nt, self.ns)
        lib().or_set_fields(self.h, _ip(f))

    def fields(self):
        f = np.zeros((self.nt, self.ns), dtype=np.int32)
        lib().or_get_fields(self.h, _ip(f))
        return f

    def engine_draws(self, n):
        out = np.zeros(n, dtype=np.uint32)
        lib().or_engine_draws(self.h, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)))
        return out

    def canonical_draws(self, n):
        out = np.zeros(n)
        lib().or_canonical_draws(self.h, n, _dp(out))
        return out

    def init(self):
        if lib().or_init(self.h) != 0:
            raise RuntimeError("or_init failed")

    def force_fields(self, target):
        """Replays a given field trajectory: during the next sweeps site (t, i) flips iff
        target[t, i] differs from its current field (None returns to Metropolis decisions)."""
        if target is None:
            lib().or_set_forced_fields(self.h, None)
        else:
            self._forced = np.ascontiguousarray(target, dtype=np.int32).reshape(self.nt, self.ns)
            lib().or_set_forced_fields(self.h, _ip(self._forced))

    def set_thermalization(self, on):
        lib().or_set_thermalization(self.h, int(on))

    def sweep(self, direction):
        if lib().or_sweep(self.h, direction) != 0:
            raise RuntimeError("or_sweep failed")

    def g(self):
        out = np.zeros((self.ns, self.ns), order="F")
        lib().or_current_g(self.h, _dp(out))
        return out

    def g_slice(self, which, t):
        out = np.zeros((self.ns, self.ns), order="F")
        if lib().or_get_g(self.h, which, t, _dp(out)) != 0:
            raise IndexError(t)
        return out

    def dyn(self):
        a = np.zeros((self.ns, self.ns), order="F")
        b = np.zeros((self.ns, self.ns), order="F")
        lib().or_current_dyn(self.h, _dp(a), _dp(b))
        return a, b

    def wrap_errors(self):
        out = np.zeros(2)
        lib().or_wrap_errors(self.h, _dp(out))
        return out

    def counts(self):
        out = np.zeros(2, dtype=np.int64)
        lib().or_counts(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
        return out

    def log_ratios(self, on=True):
        lib().or_set_ratio_log(self.h, int(on))

    def ratios(self):
        n = lib().or_ratio_log(self.h, None, 0)
        out = np.zeros(n)
        lib().or_ratio_log(self.h, _dp(out), n)
        return out

    def measure_equaltime(self):
        out = np.zeros(3)
        lib().or_measure_equaltime(self.h, _dp(out))
        return out

    def nkstars(self):
        return lib().or_nkstars(self.h)

    def measure_dynamic(self, klist=()):
        spin = np.zeros(self.nt)
        ldos = np.zeros(self.nt)
        kl = np.ascontiguousarray(klist, dtype=np.int32)
        gfk = np.zeros(max(1, len(kl)) * self.nt)
        lib().or_measure_dynamic(self.h, _dp(spin), _dp(ldos), _ip(kl), len(kl), _dp(gfk))
        return spin, ldos, gfk[: len(kl) * self.nt].reshape(len(kl), self.nt)

    def run_schedule(self, sweeps_warmup, bin_num, bin_capacity, sweeps_between_bins, equaltime=True,
                     dynamic=False, klist=()):
        kl = np.ascontiguousarray(klist, dtype=np.int32)
        eq = np.zeros((max(bin_num, 1), 3))
        spin = np.zeros((max(bin_num, 1), self.nt))
        ldos = np.zeros((max(bin_num, 1), self.nt))
        gfk = np.zeros((max(bin_num, 1), max(1, len(kl)), self.nt))
        rc = lib().or_run_schedule(self.h, sweeps_warmup, bin_num, bin_capacity, sweeps_between_bins, int(equaltime),
                                   int(dynamic), _ip(kl), len(kl), _dp(eq), _dp(spin), _dp(ldos), _dp(gfk))
        if rc != 0:
            raise RuntimeError("or_run_schedule failed")
        return {"eq": eq[:bin_num], "spin": spin[:bin_num], "ldos": ldos[:bin_num], "gfk": gfk[:bin_num, : len(kl)]}

    def stack_top(self, side):
        """(length, U S V^T of the left (0) or right (1) SVD stack)."""
        prod = np.zeros((self.ns, self.ns), order="F")
        n = lib().or_stack_top(self.h, int(side), _dp(prod))
        return n, prod

    def logdet(self):
        return lib().or_logdet(self.h)

    def logdet_grad(self):
        out = np.zeros(2 + self.ns * self.ns)
        lib().or_logdet_grad(self.h, _dp(out))
        return out[0], out[1], out[2:].reshape(self.ns, self.ns, order="F")


def set_num_threads(n):
    lib().or_set_num_threads(int(n))


def analyse(bins):
    """Mean, population stddev and stderr over the bin axis (include/observable.hpp:198-207)."""
    bins = np.asarray(bins)
    mean = bins.mean(axis=0)
    std = bins.std(axis=0)  # ddof=0, as xt::stddev
    return mean, std, std / math.sqrt(bins.shape[0])
