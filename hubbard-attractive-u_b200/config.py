"""Configuration of a DQMC run: the reference's TOML schema and parameter checks.

Mirrors DQMC::Parser::parse_toml_config (include/dqmc_parser.hpp:49-133) and
DQMC::Params (include/dqmc_params.hpp:20-45): the same keys, defaults, derived values
(ns = ng = nl^2, dt = beta / nt, bin_num divided by the number of processes) and the
same range checks (std::runtime_error there, ValueError here). An optional
[Batch] table, ignored by the reference, describes many chains for one GPU.
"""
import math
import tomllib
from dataclasses import dataclass, field

ALL_OBSERVABLES = (  # src/observable_handle.cpp:26-33
    "FillingNumber",
    "DoubleOccupation",
    "StaticSWavePairingCorrelation",
    "DynamicGreenFunctions",
    "LocalDensityOfStates",
    "LocalDynamicTransverseSpinCorrelation",
)
EQUALTIME_OBSERVABLES = ALL_OBSERVABLES[:3]
DYNAMIC_OBSERVABLES = ALL_OBSERVABLES[3:]


@dataclass
class Params:
    nl: int = 4
    ns: int = 16
    ng: int = 16
    nt: int = 160
    dt: float = 0.05
    beta: float = 8.0
    nnt: float = 1.0
    mu: float = 0.0
    u: float = 4.0
    sweeps_warmup: int = 1000
    stabilization_pace: int = 10
    momentum_list: object = "AllKstars"
    observable_list: set = field(default_factory=set)
    bin_num: int = 20
    bin_capacity: int = 100
    sweeps_between_bins: int = 10
    is_fft: bool = False
    # [Batch] (not in the reference): chains per process and their seeds
    chains: int = 1
    seed: int = 0


def _range_check(val, name, lower):
    if val < lower:
        raise ValueError(f"DQMC::Parser::range_check<T>(): '{name}' out of range.")


def parse_toml_config(source, world_size=1):
    """Parse a config (path or TOML text) into Params (include/dqmc_parser.hpp:49-133)."""
    if isinstance(source, dict):
        cfg = source
    else:
        try:
            if "\n" in source or "=" in source:
                cfg = tomllib.loads(source)
            else:
                with open(source, "rb") as f:
                    cfg = tomllib.load(f)
        except tomllib.TOMLDecodeError as err:
            raise ValueError(f"DQMC::Parser::parse_toml_config(): parsing failed.\n{err}") from err
    model = cfg.get("Model", {}).get("HubbardAttractiveU", {})
    lattice = cfg.get("Lattice", {}).get("SquareLattice", {})
    mc = cfg.get("MonteCarlo", {})
    meas = cfg.get("Measurement", {})
    p = Params()
    p.nnt = float(model.get("nnt", 1.0))
    p.u = float(model.get("u", 4.0))
    p.mu = float(model.get("mu", 0.0))
    p.nl = int(lattice.get("nl", 4))
    p.ns = p.nl * p.nl
    p.ng = p.ns
    ml = lattice.get("momentum_list", None)  # required, as in the reference (:71-86)
    if isinstance(ml, str):
        p.momentum_list = ml
    elif isinstance(ml, list) and all(isinstance(x, int) for x in ml):
        p.momentum_list = list(ml)
    else:
        raise ValueError("DQMC::Parser::parse_toml_config(): invalid input momentum list.")
    p.beta = float(mc.get("beta", 8.0))
    p.nt = int(mc.get("nt", 160))
    p.dt = p.beta / p.nt if p.nt != 0 else float("inf")  # the range check below rejects nt < 1
    p.stabilization_pace = int(mc.get("stabilization_pace", 10))
    p.is_fft = bool(mc.get("is_fft", False))
    p.sweeps_warmup = int(meas.get("sweeps_warmup", 1000))
    p.bin_num = int(math.ceil(int(meas.get("bin_num", 20)) / float(world_size)))
    p.bin_capacity = int(meas.get("bin_capacity", 100))
    p.sweeps_between_bins = int(meas.get("sweeps_between_bins", 10))
    obs = meas.get("observables")
    if not (isinstance(obs, list) and all(isinstance(x, str) for x in obs)):
        raise ValueError("DQMC::Parser::parse_toml_config(): invalid input observables.")
    is_all = "all" in obs or "All" in obs
    is_none = "none" in obs or "None" in obs
    if is_all and is_none:
        raise ValueError("DQMC::Parser::parse_toml_config(): recieved conflict observable options 'all/All' and "
                         "'none/None'.")
    if is_all:
        p.observable_list = set(ALL_OBSERVABLES)
    elif is_none:
        p.observable_list = set()
    else:
        bad = [o for o in obs if o not in ALL_OBSERVABLES]
        if bad:
            raise ValueError("Observable::Handle::initialize(): received invalid observable from the input.")
        p.observable_list = set(obs)
    batch = cfg.get("Batch", {})
    p.chains = int(batch.get("chains", 1))
    p.seed = int(batch.get("seed", 0))
    _range_check(p.u, "u", 0.0)
    _range_check(p.nl, "nl", 1)
    _range_check(p.beta, "beta", 0.0)
    _range_check(p.nt, "nt", 1)
    _range_check(p.stabilization_pace, "stabilization_pace", 1)
    _range_check(p.sweeps_warmup, "sweeps_warmup", 0)
    _range_check(p.bin_num, "bin_num", 0)
    _range_check(p.bin_capacity, "bin_capacity", 0)
    _range_check(p.sweeps_between_bins, "sweeps_between_bins", 0)
    return p


# ------------------------------------------------------------------------------------
#  Lattice momentum tables (src/square_lattice.cpp:83-118)
# ------------------------------------------------------------------------------------
def kstars(nl):
    """k points of the irreducible zone, index n -> (kx, ky) (src/square_lattice.cpp:83-95)."""
    out = []
    lo = math.ceil(nl / 2.0)
    for i in range(int(lo), nl + 1):
        for j in range(int(lo), nl + 1):
            out.append((i / nl * 2 * math.pi - math.pi, j / nl * 2 * math.pi - math.pi))
    return out


def momentum_list(nl, spec):
    """Indices of the k stars to measure (src/square_lattice.cpp:97-118,
    src/measure_handle.cpp:26-38)."""
    h = int(math.floor(nl / 2.0))
    nk = (h + 1) * (h + 1)
    if isinstance(spec, str):
        if spec == "AllKstars":
            return list(range(nk))
        if spec == "X2K2XLine":
            return [(i + 1) * h for i in range(h + 1)]
        if spec == "Gamma2MLine":
            return [i * (h + 2) for i in range(h + 1)]
        raise ValueError("Measurement::Handle::initialize(): invalid momentum list.")
    if any(k >= nk for k in spec):
        raise ValueError("Measurement::Handle::initialize(): index of momentum out of range.")
    return list(spec)


def chain_params_from(p, n_chains=None, seed=None, expk_mode=None, dynamic=None, delay_depth=0, snapshots=0):
    """hq_chain_params dictionaries of `n_chains` chains of the configuration p."""
    n = n_chains if n_chains is not None else p.chains
    s0 = seed if seed is not None else p.seed
    dyn = dynamic if dynamic is not None else bool(p.observable_list & set(DYNAMIC_OBSERVABLES))
    mode = expk_mode if expk_mode is not None else (1 if p.is_fft else -1)
    return [dict(nl=p.nl, nnt=p.nnt, u=p.u, mu=p.mu, beta=p.beta, nt=p.nt, stabilization_pace=p.stabilization_pace,
                 expk_mode=mode, seed=s0 + c, delay_depth=delay_depth, dynamic=int(dyn), snapshots=snapshots)
            for c in range(n)]
