"""Command-line driver with the reference's options and outputs (src/main.cpp:40-252).

    python hubbard-attractive-u_b200/cli.py -c config.toml -o outdir [-f ising.fields]
    torchrun --nproc-per-node G hubbard-attractive-u_b200/cli.py -c config.toml -o outdir

Runs every chain of the configuration ([Batch] chains / seed extend the reference's schema;
one chain is the reference's one MPI rank): fields from -f or seeded at random, stacks and G,
the warm-up and binned measurement schedule, then the result files of the reference
(filling.out, *.bins.out, gf.out, ..., ising.fields, momenta.out, tgrids.out).

Under torchrun (WORLD_SIZE > 1) every process owns a contiguous block of the chains on its
own GPU (LOCAL_RANK; chain c keeps seed `seed + c` whatever the process count), runs it with
no exchange, and the per-chain bins are gathered once to rank 0, which writes the files: the
reference's end-of-run gather (src/main.cpp:168-171,
include/utils/observable_gather.hpp:29-79). The bins are host arrays of a few kilobytes, so the
gather runs over gloo by default (--backend nccl gathers through the GPUs).
--checkpoint saves fields, random-engine states and bins after the run (per rank:
<path>.rank<r> under torchrun); --resume starts from such a checkpoint instead of -f.
"""
import argparse
import datetime
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


def gather_and_write(dist, outdir, params, bins, klist, fields, fields_path=None, device=None):
    """Gathers every rank's per-chain bins to rank 0 (concatenated in rank order, i.e. in global
    chain order) and writes the result files there. Returns the written paths on rank 0 and
    None elsewhere. Every rank calls it with the same observable names."""
    from hubbard_b200 import dqmc_io
    from hubbard_b200.shard import gather_bins
    pooled = gather_bins(bins, dist, device=device) if dist is not None else bins
    if dist is not None and dist.get_rank() != 0:
        return None
    return dqmc_io.write_results(outdir, params, pooled, klist, fields, fields_path=fields_path)


def main(argv=None):
    ap = argparse.ArgumentParser(description="DQMC of the attractive-U Hubbard model on a B200")
    ap.add_argument("-c", "--config", default="./example/config.toml", help="toml configuration file")
    ap.add_argument("-o", "--output", default="./example", help="folder of the result files")
    ap.add_argument("-f", "--fields", default="", help="initial Ising fields (reference field-file format)")
    ap.add_argument("--chains", type=int, default=None, help="chains of the run (default: [Batch] chains)")
    ap.add_argument("--device", type=int, default=None, help="CUDA device (default: LOCAL_RANK, else 0)")
    ap.add_argument("--backend", default="gloo", choices=["gloo", "nccl"], help="process group of the bin gather")
    ap.add_argument("--checkpoint", default="", help="save fields, random states and bins here after the run")
    ap.add_argument("--resume", default="", help="start from a checkpoint written by --checkpoint")
    args = ap.parse_args(argv)

    hq = _package()
    from hubbard_b200.config import parse_toml_config, chain_params_from
    from hubbard_b200.driver import Handle
    from hubbard_b200.shard import chains_for_rank
    from hubbard_b200 import dqmc_io

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    device = args.device if args.device is not None else local
    dist = None
    if world > 1:
        import torch.distributed as dist
        if args.backend == "nccl":
            import torch
            torch.cuda.set_device(device)
        dist.init_process_group(args.backend, timeout=datetime.timedelta(seconds=600))
    master = rank == 0

    p = parse_toml_config(args.config)
    n_total = args.chains if args.chains is not None else p.chains
    mine = chains_for_rank(n_total, rank, world)
    if not mine:
        raise SystemExit(f"rank {rank}: no chains (the run has {n_total} chains for {world} processes)")
    chains = chain_params_from(p, n_chains=n_total)[mine[0]: mine[-1] + 1]
    e = hq.Engine(chains, device=device)
    n = e.n
    ck_path = args.checkpoint + (f".rank{rank}" if world > 1 and args.checkpoint else "")
    try:
        if args.resume:
            dqmc_io.load_checkpoint(args.resume + (f".rank{rank}" if world > 1 else ""), e)
            if master:
                print(">> Configurations of ising fields and random states loaded from checkpoint.\n")
        else:
            if args.fields:
                f = dqmc_io.load_ising_fields(args.fields, p.nt, p.nl * p.nl)
                for c in range(n):
                    e.set_fields(c, f)
                if master:
                    print(">> Configurations of ising fields loaded from file.\n")
            else:
                e.fields_random()
                if master:
                    print(">> Configurations of ising fields initialized randomly.\n")
            e.init()
        if master and world > 1:
            print(f">> Distribute {n_total} chains to {world} processes.\n")
        h = Handle(e, p)
        t0 = time.perf_counter()
        h.thermalize()
        bins = h.measure()
        e.sync()
        wall = time.perf_counter() - t0
        files = gather_and_write(dist, args.output, p, bins, h.klist, e.fields(0), fields_path=args.fields or None,
                                 device=(f"cuda:{device}" if args.backend == "nccl" and dist is not None else None))
        if ck_path:
            dqmc_io.save_checkpoint(ck_path, e, bins)
        wrap = max(e.wrap_errors(c)[0] for c in range(n))
        if master:
            print(">> %d chains on %d process(es), wall time %.3f s, equal-time wrap error %.3e (rank 0)" %
                  (n_total, world, wall, wrap))
            print(">> See the results under folder '%s' (%d files)." % (args.output, len(files)))
    finally:
        e.close()
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
