"""ctypes binding of the C ABI in include/hubbard_b200.h (libhubbard_b200.so).

This is the binding a Python caller of the reference's sweep would add; every method of
`Engine` forwards to one hq_* entry point. The CUDA library is mandatory: loading fails
loudly when it is missing, and there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhubbard_b200.so")

HQ_OK = 0
HQ_E_INVALID, HQ_E_CUDA, HQ_E_NUMERIC, HQ_E_RANGE, HQ_E_NOMEM = -1, -2, -3, -4, -5
SWEEP_UP, SWEEP_DOWN, SWEEP_DYNAMIC = 0, 1, 2
SWEEP_MEASURE, SWEEP_SNAPSHOT, SWEEP_LOG_RATIOS = 1, 2, 4
G_CURRENT, G_TT, G_T0, G_0T = 0, 1, 2, 3
EXPK_DENSE, EXPK_SEPARABLE, EXPK_AUTO = 0, 1, -1

# every entry point declared in include/hubbard_b200.h
EXPORTS = [
    "hq_last_error", "hq_create", "hq_destroy", "hq_set_hopping", "hq_fields_random", "hq_set_fields",
    "hq_get_fields", "hq_init_stacks_and_g", "hq_sweep", "hq_sync", "hq_get_g", "hq_set_g",
    "hq_get_wrap_errors", "hq_get_estimators", "hq_get_estimators_all", "hq_get_dynamic_estimators", "hq_reset_estimators",
    "hq_ratio_log", "hq_logdet_adjoint", "hq_capture_graph", "hq_launch_graph", "hq_get_config",
    "hq_upload_fields_i8", "hq_download_fields_i8", "hq_get_stream", "hq_profile_enable", "hq_profile_collect",
    "hq_equaltime_g_noalloc", "hq_autotune", "hq_get_stack", "hq_get_rng_state", "hq_set_rng_state",
    "hq_set_sweep_mode", "hq_get_sweep_mode", "hq_phase_cycles",
]
PROFILE_CLASSES = ["interval", "bchain", "udt", "gemm", "invert", "measure", "dynamic", "adjoint", "interval_cluster",
                   "sweep"]
SWEEP_LAUNCHES, SWEEP_PERSISTENT = 0, 1
SWEEP_PHASE_CLOCKS = 8
PHASES = ["wait", "interval", "bchain", "udt", "push_gemm", "builder_gemm_12", "invert", "builder_gemm_34", "measure",
          "items"]


class HqChainParams(ctypes.Structure):
    _fields_ = [
        ("nl", ctypes.c_int),
        ("nnt", ctypes.c_double),
        ("u", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("beta", ctypes.c_double),
        ("nt", ctypes.c_int),
        ("stabilization_pace", ctypes.c_int),
        ("expk_mode", ctypes.c_int),
        ("seed", ctypes.c_longlong),
        ("delay_depth", ctypes.c_int),
        ("dynamic", ctypes.c_int),
        ("snapshots", ctypes.c_int),
    ]


class HqTuneEntry(ctypes.Structure):
    _fields_ = [
        ("nl", ctypes.c_int),
        ("expk_mode", ctypes.c_int),
        ("delay_depth", ctypes.c_int),
        ("ms_per_sweep", ctypes.c_double),
        ("chosen", ctypes.c_int),
        ("cluster_size", ctypes.c_int),
        ("sweep_mode", ctypes.c_int),
    ]


class HqError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None


def lib():
    """Load libhubbard_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with hubbard-attractive-u_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        c_int, c_dbl, c_ll, vp = ctypes.c_int, ctypes.c_double, ctypes.c_longlong, ctypes.c_void_p
        dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        sig = {
            "hq_last_error": [ctypes.c_char_p, ctypes.c_size_t],
            "hq_create": [c_int, c_int, ctypes.POINTER(HqChainParams), ctypes.POINTER(vp)],
            "hq_destroy": [vp],
            "hq_set_hopping": [vp, c_int, dp],
            "hq_fields_random": [vp, c_int],
            "hq_set_fields": [vp, c_int, ip],
            "hq_get_fields": [vp, c_int, ip],
            "hq_init_stacks_and_g": [vp],
            "hq_sweep": [vp, c_int, c_int],
            "hq_sync": [vp],
            "hq_get_g": [vp, c_int, c_int, c_int, dp],
            "hq_set_g": [vp, c_int, dp],
            "hq_get_wrap_errors": [vp, c_int, dp],
            "hq_get_estimators": [vp, c_int, dp],
            "hq_get_estimators_all": [vp, dp],
            "hq_get_dynamic_estimators": [vp, c_int, dp, dp, dp],
            "hq_reset_estimators": [vp, c_int],
            "hq_ratio_log": [vp, c_int, c_ll, dp, c_ll, ctypes.POINTER(c_ll)],
            "hq_logdet_adjoint": [vp, dp, dp],
            "hq_capture_graph": [vp, c_int, c_int],
            "hq_launch_graph": [vp, c_int],
            "hq_get_config": [vp, c_int, ip, ip],
            "hq_upload_fields_i8": [vp, ctypes.c_void_p],
            "hq_download_fields_i8": [vp, ctypes.c_void_p],
            "hq_get_stream": [vp, ctypes.POINTER(vp)],
            "hq_profile_enable": [vp, c_int],
            "hq_profile_collect": [vp, dp, ctypes.POINTER(c_ll), c_int],
            "hq_equaltime_g_noalloc": [c_int, c_dbl, c_dbl, c_dbl, c_dbl, c_int, c_int, vp, vp, vp],
            "hq_autotune": [vp, c_int, ctypes.POINTER(HqTuneEntry), c_int, ip],
            "hq_get_stack": [vp, c_int, c_int, ip, dp, dp, dp],
            "hq_get_rng_state": [vp, c_int, ctypes.POINTER(ctypes.c_uint)],
            "hq_set_rng_state": [vp, c_int, ctypes.c_uint],
            "hq_set_sweep_mode": [vp, c_int],
            "hq_get_sweep_mode": [vp, ip],
            "hq_phase_cycles": [vp, ctypes.POINTER(ctypes.c_ulonglong), c_int, c_int],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = c_int
        _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(4096)
    lib().hq_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(rc):
    if rc != HQ_OK:
        raise HqError(rc, last_error())


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Engine:
    """A context of independent Markov chains on one GPU (one `hq_ctx`)."""

    def __init__(self, chains, device=0):
        self.params = list(chains)
        arr = (HqChainParams * len(self.params))()
        for k, p in enumerate(self.params):
            arr[k] = HqChainParams(int(p["nl"]), float(p.get("nnt", 1.0)), float(p.get("u", 4.0)),
                                   float(p.get("mu", 0.0)), float(p.get("beta", 8.0)), int(p.get("nt", 160)),
                                   int(p.get("stabilization_pace", 10)), int(p.get("expk_mode", EXPK_AUTO)),
                                   int(p.get("seed", 0)), int(p.get("delay_depth", 0)), int(p.get("dynamic", 0)),
                                   int(p.get("snapshots", 0)))
        h = ctypes.c_void_p()
        check(lib().hq_create(int(device), len(self.params), arr, ctypes.byref(h)))
        self.h = h
        self.n = len(self.params)

    def close(self):
        if getattr(self, "h", None):
            lib().hq_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _N(self, c):
        return int(self.params[c]["nl"]) ** 2

    def _nt(self, c):
        return int(self.params[c].get("nt", 160))

    def set_hopping(self, chain, hop):
        hop = np.asfortranarray(hop, dtype=np.float64)
        check(lib().hq_set_hopping(self.h, chain, _dp(hop)))

    def fields_random(self, chain=None):
        for c in (range(self.n) if chain is None else [chain]):
            check(lib().hq_fields_random(self.h, c))

    def set_fields(self, chain, f):
        f = np.ascontiguousarray(f, dtype=np.int32)
        check(lib().hq_set_fields(self.h, chain, _ip(f)))

    def fields(self, chain):
        f = np.zeros((self._nt(chain), self._N(chain)), dtype=np.int32)
        check(lib().hq_get_fields(self.h, chain, _ip(f)))
        return f

    def init(self):
        check(lib().hq_init_stacks_and_g(self.h))

    def sweep(self, direction, flags=0):
        check(lib().hq_sweep(self.h, int(direction), int(flags)))

    def sync(self):
        check(lib().hq_sync(self.h))

    def g(self, chain, which=G_CURRENT, slice_=0):
        N = self._N(chain)
        out = np.zeros((N, N), order="F")
        check(lib().hq_get_g(self.h, chain, which, slice_, _dp(out)))
        return out

    def set_g(self, chain, g):
        g = np.asfortranarray(g, dtype=np.float64)
        check(lib().hq_set_g(self.h, chain, _dp(g)))

    def wrap_errors(self, chain):
        out = np.zeros(2)
        check(lib().hq_get_wrap_errors(self.h, chain, _dp(out)))
        return out

    def estimators(self, chain):
        out = np.zeros(6)
        check(lib().hq_get_estimators(self.h, chain, _dp(out)))
        return out

    def estimators_all(self):
        """The six estimator sums of every chain as an (n_chains, 6) array, one copy."""
        out = np.zeros((self.n, 6))
        check(lib().hq_get_estimators_all(self.h, _dp(out)))
        return out

    def dynamic_estimators(self, chain):
        nt, N = self._nt(chain), self._N(chain)
        spin, ldos, gd = np.zeros(nt), np.zeros(nt), np.zeros((N, nt))
        check(lib().hq_get_dynamic_estimators(self.h, chain, _dp(spin), _dp(ldos), _dp(gd)))
        return spin, ldos, gd

    def reset_estimators(self, reset_wrap=False):
        check(lib().hq_reset_estimators(self.h, int(reset_wrap)))

    def ratio_log(self, chain, capacity=0):
        cnt = ctypes.c_longlong(0)
        check(lib().hq_ratio_log(self.h, chain, int(capacity), None, 0, ctypes.byref(cnt)))
        out = np.zeros(max(cnt.value, 0))
        if cnt.value > 0:
            check(lib().hq_ratio_log(self.h, chain, 0, _dp(out), cnt.value, ctypes.byref(cnt)))
        return out

    def logdet_adjoint(self):
        tot = sum(2 + self._N(c) ** 2 for c in range(self.n))
        out = np.zeros(tot)
        ld = np.zeros(self.n)
        check(lib().hq_logdet_adjoint(self.h, _dp(out), _dp(ld)))
        res, off = [], 0
        for c in range(self.n):
            N = self._N(c)
            res.append((out[off], out[off + 1], out[off + 2: off + 2 + N * N].reshape(N, N, order="F")))
            off += 2 + N * N
        return ld, res

    def capture_graph(self, direction, flags=0):
        check(lib().hq_capture_graph(self.h, int(direction), int(flags)))

    def launch_graph(self, direction):
        check(lib().hq_launch_graph(self.h, int(direction)))

    def config(self, chain):
        m, k = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().hq_get_config(self.h, chain, ctypes.byref(m), ctypes.byref(k)))
        return m.value, k.value

    def set_sweep_mode(self, mode):
        """SWEEP_PERSISTENT (one persistent launch per sweep) or SWEEP_LAUNCHES (one launch per
        phase and interval); drops the captured sweep graphs."""
        check(lib().hq_set_sweep_mode(self.h, int(mode)))

    def phase_cycles(self, reset=False):
        """Cycles per phase of the persistent sweeps run with SWEEP_PHASE_CLOCKS (dict over PHASES)."""
        buf = (ctypes.c_ulonglong * len(PHASES))()
        check(lib().hq_phase_cycles(self.h, buf, len(PHASES), int(reset)))
        return dict(zip(PHASES, (int(v) for v in buf)))

    def sweep_mode(self):
        m = ctypes.c_int(0)
        check(lib().hq_get_sweep_mode(self.h, ctypes.byref(m)))
        return m.value

    def autotune(self, sweeps=2):
        """Times every (expK mode, delay depth) candidate per lattice size on whole sweeps and
        keeps the fastest, then the two sweep modes (entries with nl = 0); the chains' state is
        restored after each candidate. Returns the timed candidates as dicts."""
        cap = 64
        buf = (HqTuneEntry * cap)()
        n = ctypes.c_int(0)
        check(lib().hq_autotune(self.h, int(sweeps), buf, cap, ctypes.byref(n)))
        return [dict(nl=e.nl, expk_mode=e.expk_mode, delay_depth=e.delay_depth, ms_per_sweep=e.ms_per_sweep,
                     chosen=bool(e.chosen), cluster_size=e.cluster_size, sweep_mode=e.sweep_mode)
                for e in buf[:min(n.value, cap)]]

    def stack(self, chain, side):
        """(length, U, D, V) of the top of a chain's left (0) or right (1) UDV stack; the
        product of all pushes is U diag(D) V^T. U, D, V are None for an empty stack."""
        N = self._N(chain)
        n = ctypes.c_int(0)
        check(lib().hq_get_stack(self.h, chain, side, ctypes.byref(n), None, None, None))
        if n.value == 0:
            return 0, None, None, None
        U, V, D = np.zeros((N, N), order="F"), np.zeros((N, N), order="F"), np.zeros(N)
        check(lib().hq_get_stack(self.h, chain, side, ctypes.byref(n), _dp(U), _dp(D), _dp(V)))
        return n.value, U, D, V

    def rng_state(self, chain):
        v = ctypes.c_uint(0)
        check(lib().hq_get_rng_state(self.h, chain, ctypes.byref(v)))
        return v.value

    def set_rng_state(self, chain, state):
        check(lib().hq_set_rng_state(self.h, chain, int(state)))

    def stream(self):
        s = ctypes.c_void_p()
        check(lib().hq_get_stream(self.h, ctypes.byref(s)))
        return s.value

    def profile_enable(self, on=True):
        check(lib().hq_profile_enable(self.h, int(on)))

    def profile_collect(self, ms, counts):
        """Adds the per-class launch times (ms) and counts of the most recent sweep."""
        check(lib().hq_profile_collect(self.h, _dp(ms), counts.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                                       len(ms)))

    def upload_fields_i8(self, buf):
        check(lib().hq_upload_fields_i8(self.h, ctypes.c_void_p(buf)))

    def download_fields_i8(self, buf):
        check(lib().hq_download_fields_i8(self.h, ctypes.c_void_p(buf)))
