"""Command-line driver with the reference's options and outputs (src/main.cpp:40-252).

    python hubbard-attractive-u_b200/cli.py -c config.toml -o outdir [-f ising.fields]

Runs every chain of the configuration on one GPU ([Batch] chains / seed extend the reference's
schema; one chain is the reference's one MPI rank): fields from -f or seeded at random,
stacks and G, the warm-up and binned measurement schedule, then the result files of the
reference (filling.out, *.bins.out, gf.out, ..., ising.fields, momenta.out, tgrids.out).
--checkpoint saves fields, random-engine states and bins after the run; --resume starts from
such a checkpoint instead of -f.
"""
import argparse
import os
import sys
import time


def _package():
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    if root not in sys.path:
        sys.path.insert(0, root)
    from __graft_entry__ import load_package
    return load_package()


def main(argv=None):
    ap = argparse.ArgumentParser(description="DQMC of the attractive-U Hubbard model on a B200")
    ap.add_argument("-c", "--config", default="./example/config.toml", help="toml configuration file")
    ap.add_argument("-o", "--output", default="./example", help="folder of the result files")
    ap.add_argument("-f", "--fields", default="", help="initial Ising fields (reference field-file format)")
    ap.add_argument("--chains", type=int, default=None, help="chains on this GPU (default: [Batch] chains)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--checkpoint", default="", help="save fields, random states and bins here after the run")
    ap.add_argument("--resume", default="", help="start from a checkpoint written by --checkpoint")
    args = ap.parse_args(argv)

    hq = _package()
    from hubbard_b200.config import parse_toml_config, chain_params_from
    from hubbard_b200.driver import Handle
    from hubbard_b200 import dqmc_io

    p = parse_toml_config(args.config)
    n = args.chains if args.chains is not None else p.chains
    e = hq.Engine(chain_params_from(p, n_chains=n), device=args.device)
    try:
        if args.resume:
            dqmc_io.load_checkpoint(args.resume, e)
            print(">> Configurations of ising fields and random states loaded from checkpoint.\n")
        else:
            if args.fields:
                f = dqmc_io.load_ising_fields(args.fields, p.nt, p.nl * p.nl)
                for c in range(n):
                    e.set_fields(c, f)
                print(">> Configurations of ising fields loaded from file.\n")
            else:
                e.fields_random()
                print(">> Configurations of ising fields initialized randomly.\n")
            e.init()
        h = Handle(e, p)
        t0 = time.perf_counter()
        h.thermalize()
        bins = h.measure()
        e.sync()
        wall = time.perf_counter() - t0
        files = dqmc_io.write_results(args.output, p, bins, h.klist, e.fields(0), fields_path=args.fields or None)
        if args.checkpoint:
            dqmc_io.save_checkpoint(args.checkpoint, e, bins)
        print(">> %d chains, wall time %.3f s, equal-time wrap error %.3e" %
              (n, wall, max(e.wrap_errors(c)[0] for c in range(n))))
        print(">> See the results under folder '%s' (%d files)." % (args.output, len(files)))
    finally:
        e.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
