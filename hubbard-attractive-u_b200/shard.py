"""Chain sharding across GPUs and the end-of-run gather of the bins.

The reference runs one Markov chain per MPI rank and gathers every rank's bins to rank 0
once at the end (include/utils/observable_gather.hpp:29-79, Boost.MPI isend/irecv). Here
every GPU process owns a contiguous block of chains (no exchange during the run) and the
per-chain bin arrays are gathered once with torch.distributed (NCCL between GPUs, gloo on
CPU).
"""
import numpy as np


def chains_for_rank(n_total, rank, world):
    """Contiguous, balanced block of chain indices of `rank` (chains are independent)."""
    base, extra = divmod(n_total, world)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return list(range(lo, hi))


def gather_bins(bins, dist, device=None):
    """Gathers {name: array [chains, bins, ...]} of every rank onto rank 0 (concatenated
    along the chain axis in rank order); other ranks get None. Every rank calls it with
    the same observable names."""
    import torch
    rank, world = dist.get_rank(), dist.get_world_size()
    out = {}
    for name in sorted(bins):
        a = np.ascontiguousarray(bins[name], dtype=np.float64)
        t = torch.from_numpy(a)
        if device is not None:
            t = t.to(device)
        n = torch.tensor([a.shape[0]], dtype=torch.int64, device=t.device)
        sizes = [torch.zeros_like(n) for _ in range(world)]
        dist.all_gather(sizes, n)
        nmax = int(max(s.item() for s in sizes))
        pad = torch.zeros((nmax,) + tuple(a.shape[1:]), dtype=t.dtype, device=t.device)
        pad[: a.shape[0]] = t
        parts = [torch.zeros_like(pad) for _ in range(world)]
        dist.all_gather(parts, pad)
        if rank == 0:
            out[name] = np.concatenate([p[: int(s.item())].cpu().numpy() for p, s in zip(parts, sizes)], axis=0)
    return out if rank == 0 else None
