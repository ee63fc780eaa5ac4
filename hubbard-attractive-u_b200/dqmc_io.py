"""Result files, field files and checkpoints.

The writers produce the reference's text formats (include/dqmc_io.hpp:130-289, called from
src/main.cpp:182-249): integer columns "%| 15d|", value columns "%| 30.15f|" (time grids
"%| 30.8f|"), a header line of dimensions, then one row per element in row-major order.
Checkpoints (not in the reference, which saves only the fields) also keep every chain's
random-engine state and the bins measured so far, so that a run continues exactly.
"""
import os

import numpy as np

from .config import kstars
from .driver import analyse

# observable name -> file stem (src/main.cpp:188-236)
OUTPUT_STEMS = {
    "FillingNumber": "filling",
    "DoubleOccupation": "double_occu",
    "DynamicGreenFunctions": "gf",
    "LocalDensityOfStates": "ldos",
    "StaticSWavePairingCorrelation": "swave_corr",
    "LocalDynamicTransverseSpinCorrelation": "spin_corr",
}


def _i(v):
    return "{: 15d}".format(int(v))


def _f(v, prec=15):
    return "{: 30.{}f}".format(float(v), prec)


def print_observable(f, mean, std, err, show_header=True):
    """Mean, population stddev and stderr of an observable (include/dqmc_io.hpp:130-173)."""
    mean, std, err = np.asarray(mean), np.asarray(std), np.asarray(err)
    if mean.ndim == 0:
        if show_header:
            f.write(_i(1) + "\n")
        f.write(_i(0) + _f(mean) + _f(std) + _f(err) + "\n")
        return
    if show_header:
        f.write("".join(_i(d) for d in mean.shape) + "\n")
    for idx in np.ndindex(mean.shape):
        f.write("".join(_i(i) for i in idx) + _f(mean[idx]) + _f(std[idx]) + _f(err[idx]) + "\n")


def print_observable_data(f, bins, show_header=True):
    """Per-bin values, bin index first (include/dqmc_io.hpp:175-205)."""
    bins = np.asarray(bins)
    if show_header:
        f.write("".join(_i(d) for d in bins.shape) + "\n")
    for idx in np.ndindex(bins.shape):
        f.write("".join(_i(i) for i in idx) + _f(bins[idx]) + "\n")


def save_ising_fields(path, fields):
    """nt ns, then one "t i s" row per field (include/dqmc_io.hpp:214-232)."""
    fields = np.asarray(fields)
    nt, ns = fields.shape
    with open(path, "w") as f:
        f.write(_i(nt) + _i(ns) + "\n")
        for t in range(nt):
            for i in range(ns):
                f.write(_i(t) + _i(i) + _i(fields[t, i]) + "\n")


def load_ising_fields(path, nt, ns):
    """Reads a field file; its dimensions must be (nt, ns) (include/dqmc_io.hpp:234-255)."""
    with open(path) as f:
        head = f.readline().split()
        if len(head) < 2 or int(head[0]) != nt or int(head[1]) != ns:
            raise ValueError("load_ising_fields: contradictory dimensions of the ising fields.")
        out = np.zeros((nt, ns), dtype=np.int32)
        for line in f:
            parts = line.split()
            if len(parts) >= 3:
                out[int(parts[0]), int(parts[1])] = int(parts[2])
    if not np.all(np.abs(out) == 1):
        raise ValueError("load_ising_fields: every field must be +1 or -1")
    return out


def print_momentum_list(f, nl, klist):
    """nk nkstars, then "k index kx ky" (include/dqmc_io.hpp:262-276)."""
    ks = kstars(nl)
    f.write(_i(len(klist)) + _i(len(ks)) + "\n")
    for k, idx in enumerate(klist):
        kx, ky = ks[idx]
        f.write(_i(k) + _i(idx) + _f(kx) + _f(ky) + "\n")


def print_imaginary_time_grids(f, nt, beta, dt):
    """nt beta dt, then "t tau" (include/dqmc_io.hpp:278-289)."""
    f.write(_i(nt) + _f(beta, 8) + _f(dt, 8) + "\n")
    for t in range(nt):
        f.write(_i(t) + _f(t * dt, 8) + "\n")


def write_results(outdir, params, bins, klist, fields, fields_path=None):
    """Every result file of src/main.cpp:182-249 under outdir. bins: observable name ->
    [chain][bin][...] (driver.Handle.measure); chains are pooled as the reference pools the
    bins of its MPI ranks. fields: the (nt, N) fields written to ising.fields (or to
    fields_path, the file the run was started from)."""
    os.makedirs(outdir, exist_ok=True)
    written = []
    for name, stem in OUTPUT_STEMS.items():
        if name not in bins or name not in params.observable_list:
            continue
        data = np.asarray(bins[name])
        data = data.reshape((-1,) + data.shape[2:])
        mean, std, err = analyse(data)
        for suffix, fn in ((".out", lambda f: print_observable(f, mean, std, err)),
                           (".bins.out", lambda f: print_observable_data(f, data))):
            path = os.path.join(outdir, stem + suffix)
            with open(path, "w") as f:
                fn(f)
            written.append(path)
    fpath = fields_path or os.path.join(outdir, "ising.fields")
    save_ising_fields(fpath, fields)
    written.append(fpath)
    for stem, fn in (("momenta.out", lambda f: print_momentum_list(f, params.nl, klist)),
                     ("tgrids.out", lambda f: print_imaginary_time_grids(f, params.nt, params.beta, params.dt))):
        path = os.path.join(outdir, stem)
        with open(path, "w") as f:
            fn(f)
        written.append(path)
    return written


def save_checkpoint(path, engine, bins=None, meta=None):
    """Fields and random-engine state of every chain, plus any bins (npz). The engine must be
    between round trips (stacks at tau = 0)."""
    n = engine.n
    arrays = {"fields": np.stack([engine.fields(c).astype(np.int8) for c in range(n)]),
              "rng": np.array([engine.rng_state(c) for c in range(n)], dtype=np.uint32)}
    for name, b in (bins or {}).items():
        arrays["bins_" + name] = np.asarray(b)
    for k, v in (meta or {}).items():
        arrays["meta_" + k] = np.asarray(v)
    np.savez(path, **arrays)


def load_checkpoint(path, engine):
    """Restores fields and random-engine states into an engine of the same chains and
    rebuilds its stacks and G; returns (bins, meta)."""
    z = np.load(path)
    fields, rng = z["fields"], z["rng"]
    if fields.shape[0] != engine.n:
        raise ValueError("load_checkpoint: the checkpoint holds %d chains, the engine %d" % (fields.shape[0], engine.n))
    for c in range(engine.n):
        engine.set_fields(c, fields[c].astype(np.int32))
        engine.set_rng_state(c, int(rng[c]))
    engine.init()
    bins = {k[5:]: z[k] for k in z.files if k.startswith("bins_")}
    meta = {k[5:]: z[k] for k in z.files if k.startswith("meta_")}
    return bins, meta
