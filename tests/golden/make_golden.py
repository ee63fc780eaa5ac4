"""Generates the golden fixtures of the tests from the reference's own example run.

Reads JefferyWangSH/hubbard-attractive-U's `example/` directory (config.toml, the binned
observables *.out / *.bins.out, log.out and the final Ising field configuration
ising.fields) and writes:
  example_run.json     : observables (mean, stddev, stderr, per-bin values), wrap errors
  example_fields.txt   : the final field configuration, "nt ns" then nt rows of ns +-1
  example_config.toml  : the run's configuration file (verbatim)
  example_format.json  : verbatim lines of momenta.out, tgrids.out, ising.fields and of the
                         binned output files (format checks of the result writers)
Usage: python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def read_table(path):
    rows = []
    for ln in open(path):
        parts = ln.split()
        if parts:
            rows.append([float(x) for x in parts])
    return rows


def main(ref):
    ex = os.path.join(ref, "example")
    out = {"source": "example/ of the reference (4 MPI ranks, L=4, beta=8, nt=160, 20 bins)"}
    scalars = {"filling": "filling", "double_occupancy": "double_occu", "swave": "swave_corr"}
    for key, stem in scalars.items():
        r = read_table(os.path.join(ex, stem + ".out"))[0]
        bins = [row[1] for row in read_table(os.path.join(ex, stem + ".bins.out"))]
        out[key] = {"mean": r[1], "stddev": r[2], "stderr": r[3], "bins": bins}
    for key, stem in {"spin_corr": "spin_corr", "ldos": "ldos"}.items():
        rows = read_table(os.path.join(ex, stem + ".out"))
        out[key] = {"mean": [r[1] for r in rows], "stderr": [r[3] for r in rows]}
    rows = read_table(os.path.join(ex, "gf.out"))
    nk = int(max(r[0] for r in rows)) + 1
    nt = int(max(r[1] for r in rows)) + 1
    out["gf"] = {"nk": nk, "nt": nt, "mean": [r[2] for r in rows], "stderr": [r[4] for r in rows]}
    mom = read_table(os.path.join(ex, "momenta.out"))
    out["momenta"] = [[int(r[1]), r[2], r[3]] for r in mom[1:]]
    log = open(os.path.join(ex, "log.out")).read()
    m = re.search(r"wrapping error: ([0-9.eE+-]+) \(equal-time\) and ([0-9.eE+-]+) \(dynamic\)", log)
    out["wrap_error"] = {"equaltime": float(m.group(1)), "dynamic": float(m.group(2))}
    with open(os.path.join(HERE, "example_run.json"), "w") as f:
        json.dump(out, f, indent=1)
    # fields: header "nt ns" then lines "t i s"
    lines = open(os.path.join(ex, "ising.fields")).read().split("\n")
    nt_, ns_ = (int(x) for x in lines[0].split())
    f = [[0] * ns_ for _ in range(nt_)]
    for ln in lines[1:]:
        p = ln.split()
        if len(p) == 3:
            f[int(p[0])][int(p[1])] = int(p[2])
    with open(os.path.join(HERE, "example_fields.txt"), "w") as g:
        g.write(f"{nt_} {ns_}\n")
        for row in f:
            g.write(" ".join("%d" % v for v in row) + "\n")
    with open(os.path.join(ex, "config.toml")) as src, open(os.path.join(HERE, "example_config.toml"), "w") as dst:
        dst.write(src.read())
    # verbatim lines of the output files, for the writers' format checks
    fmt = {}
    for name, nlines in (("momenta.out", None), ("tgrids.out", None), ("ising.fields", 6), ("filling.bins.out", 5),
                         ("gf.bins.out", 5), ("spin_corr.bins.out", 5), ("gf.out", 3)):
        lines = open(os.path.join(ex, name)).read().split("\n")
        lines = [ln for ln in lines if ln.strip()]
        fmt[name] = lines if nlines is None else lines[:nlines]
    with open(os.path.join(HERE, "example_format.json"), "w") as f:
        json.dump(fmt, f, indent=0)
    print("wrote example_run.json, example_fields.txt, example_config.toml, example_format.json")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
