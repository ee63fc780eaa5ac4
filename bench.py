#!/usr/bin/env python
"""Throughput of the batched DQMC sweep on B200.

Workload (the metric's configuration): 256 independent Markov chains of the attractive-U
Hubbard model on a 12x12 periodic lattice (N = 144), t = 1, |U| = 4, mu = 0, beta = 10,
dt = 0.1 (nt = 100 slices), stabilisation every 10 slices, Ising fields i.i.d. +-1 from
per-chain seeds 1000 + c (the reference's minstd_rand0 stream). One step = one
directional update sweep (the reference's unit, src/dqmc_handle.cpp:72) of every chain,
alternating 0 -> beta and beta -> 0, with the fused equal-time estimators on.

  value : aggregate directional sweeps/s with the chains resident in HBM (CUDA events
          on the library's stream around K captured-graph sweeps, max over ranks)
  e2e   : the same metric through the C ABI from host buffers: per step, the fields
          are copied host -> device, the stacks and G are built (hq_init_stacks_and_g),
          one sweep runs, and fields + estimator sums are copied back.
  --impl reference : the CPU restatement of the reference path (oracle/) on all host
          cores, one chain per process, same configuration and unit.

Multi-GPU (torchrun): every rank runs its own 256 chains (weak scaling, no collective
in the data path); the elapsed time is the max over ranks.
"""
import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sweeps/s @12x12 β=10: 256 batched chains vs 1-chain GPU; G err≤1e-10"
CFG = dict(nl=12, nnt=1.0, u=4.0, mu=0.0, beta=10.0, nt=100, stabilization_pace=10)
N_CHAINS = 256
SEED0 = 1000


def chain_params(rank, n=N_CHAINS, expk_mode=-1):
    """The metric's chains: seeds 1000 + c, c counted across ranks."""
    return [dict(CFG, seed=SEED0 + rank * n + c, expk_mode=expk_mode) for c in range(n)]


# --------------------------------------------------------------------------------------
#  CPU legs (the oracle is the checker and the timed CPU baseline only)
# --------------------------------------------------------------------------------------
def _cpu_worker(args):
    seed, warm, steps, budget_s = args
    from oracle.oracle import OracleChain, set_num_threads, UP, DOWN
    set_num_threads(1)
    ch = OracleChain(CFG["nl"], nnt=CFG["nnt"], u=CFG["u"], mu=CFG["mu"], beta=CFG["beta"], nt=CFG["nt"],
                     pace=CFG["stabilization_pace"], seed=seed)
    ch.fields_random()
    ch.init()
    d = UP
    for _ in range(warm):
        ch.sweep(d)
        d = DOWN if d == UP else UP
    t0 = time.perf_counter()
    done = 0
    while done < steps or (steps == 0 and time.perf_counter() - t0 < budget_s):
        ch.sweep(d)
        d = DOWN if d == UP else UP
        done += 1
        if budget_s and time.perf_counter() - t0 > budget_s and done >= 2 and steps == 0:
            break
    return done, time.perf_counter() - t0


def cpu_throughput(procs, warm, steps, budget_s):
    """Aggregate directional sweeps/s of `procs` single-threaded oracle chains."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(SEED0 + p, warm, steps, budget_s) for p in range(procs)])
    total = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    return total / wall, total, wall


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    procs = os.cpu_count() or 1
    steps = max(2, args.steps)
    thr, total, wall = cpu_throughput(procs, max(1, args.warmup), steps, 0)
    line = {
        "metric": METRIC, "impl": "reference", "value": thr, "unit": "sweeps/s", "n_gpus": 0, "steps": steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * wall / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Ising fields, minstd_rand0)",
        "config": {"workload": "DQMC update sweeps, 12x12 lattice, beta=10, nt=100, pace 10, one chain per host core",
                   "chains": procs, **CFG},
        "cpu_baseline": {"value": thr, "unit": "sweeps/s", "cores": procs, "kind": "port",
                         "sample": f"{procs} processes x {steps} directional sweeps of one 12x12 chain each "
                                   f"(OpenBLAS 1 thread each)"},
        "e2e": {"value": thr, "unit": "sweeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------------------
#  GPU leg
# --------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if not self.proc:
            return out
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for ln in open(self.path):
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sms.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
            os.unlink(self.path)
        except Exception:
            pass
        out["sm_mhz"] = statistics.median(sms) if sms else None
        out["sm_max_mhz"] = mx
        out["reasons"] = sorted(reasons)
        out["samples"] = len(sms)
        return out


def fp64_peak_tflops(torch, device):
    """cuBLAS DGEMM throughput (8192^3, best of 5) on this GPU: the FP64 roofline peak."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def interval_flops(nl, n_slices, accepted, kmax, expk_mode):
    """Algorithmic FP64 flops of the interval kernel: wraps of n_slices slices plus
    `accepted` flips in submatrix form (blocks of kmax sites): per flip the rank-1 share of
    the DMMA flush (2 N^2) and its panel row / column (4 N m for the m-th flip of a block)."""
    N = nl * nl
    wrap = (8.0 * N * nl ** 3) if expk_mode == 1 else (4.0 * N ** 3)  # two expK applications per slice
    blocks = n_slices * ((N + kmax - 1) // kmax)
    per_block = accepted / blocks if blocks else 0.0
    mbar = max(per_block - 1.0, 0.0) / 2.0  # mean in-block index of an accepted flip
    flip = 2.0 * N * N + 4.0 * N * mbar
    return n_slices * wrap + accepted * flip


def run_gpu(args):
    import numpy as np
    import torch
    from __graft_entry__ import load_package
    hq = load_package()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    n = args.chains
    peak = fp64_peak_tflops(torch, local) if not args.no_peak else None

    eng = hq.Engine(chain_params(rank, n), device=local)
    eng.fields_random()
    eng.init()
    # expK application and delay depth picked by timing (the chains' state is restored)
    tune = [] if args.no_tune else eng.autotune(sweeps=1)
    expk_mode, kmax = eng.config(0)
    stream = torch.cuda.ExternalStream(eng.stream())
    # warm-up: W directional sweeps (alternating), then capture one graph per direction
    d = hq.SWEEP_UP
    for _ in range(max(args.warmup, 3)):
        eng.sweep(d, hq.SWEEP_MEASURE)
        d = hq.SWEEP_DOWN if d == hq.SWEEP_UP else hq.SWEEP_UP
    eng.sync()
    eng.profile_enable(True)
    eng.capture_graph(hq.SWEEP_UP, hq.SWEEP_MEASURE)
    eng.capture_graph(hq.SWEEP_DOWN, hq.SWEEP_MEASURE)
    # one untimed replay of each direction
    for _ in range(2):
        eng.sweep(d, hq.SWEEP_MEASURE)
        d = hq.SWEEP_DOWN if d == hq.SWEEP_UP else hq.SWEEP_UP
    eng.sync()
    eng.reset_estimators(reset_wrap=True)
    acc0 = np.array([eng.estimators(c) for c in range(n)])

    ms_cls = np.zeros(len(hq.capi.PROFILE_CLASSES))
    cnt_cls = np.zeros(len(hq.capi.PROFILE_CLASSES), dtype=np.int64)
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        eng.sweep(d, hq.SWEEP_MEASURE)
        eng.profile_collect(ms_cls, cnt_cls)  # waits for the sweep; adds its per-launch event times
        d = hq.SWEEP_DOWN if d == hq.SWEEP_UP else hq.SWEEP_UP
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    acc1 = np.array([eng.estimators(c) for c in range(n)])
    accepted = float((acc1[:, 5] - acc0[:, 5]).sum())
    proposed = float((acc1[:, 4] - acc0[:, 4]).sum())
    wrap = max(eng.wrap_errors(c)[0] for c in range(n))
    value = world * n * args.steps / (ms * 1e-3)

    # roofline of the dominant kernel class (largest share of device time)
    dom = int(np.argmax(ms_cls))
    dom_name = hq.capi.PROFILE_CLASSES[dom]
    avg_launch_ms = ms_cls[dom] / max(1, cnt_cls[dom])
    if dom_name == "interval":
        flops_total = interval_flops(CFG["nl"], n * CFG["nt"] * args.steps, accepted, kmax, expk_mode)
        flops_per_launch = flops_total / max(1, cnt_cls[dom])
    else:
        flops_per_launch = None
    achieved = (flops_per_launch / (avg_launch_ms * 1e-3) / 1e12) if flops_per_launch else None
    # DRAM bytes of one k_interval launch: ncu capture of a 16-chain launch (2.864 MB read, 0
    # written), scaled by the chains of one launch here (the traffic is per-chain state; with
    # two chain groups a launch covers half of the chains)
    chains_per_launch = n * (CFG["nt"] // CFG["stabilization_pace"]) * args.steps / max(1, int(cnt_cls[dom]))
    traffic = 2.864e6 * chains_per_launch / 16 if dom_name == "interval" else None
    # the whole sweep in the dense-GEMM flop convention (6N^3 per slice, 2N^2 per accepted flip,
    # 33N^3 per stabilisation), over the measured step time
    N = CFG["nl"] ** 2
    n_stab = -(-CFG["nt"] // CFG["stabilization_pace"])
    f_sweep = world * (n * args.steps * (CFG["nt"] * 6.0 * N ** 3 + n_stab * 33.0 * N ** 3) + accepted * 2.0 * N ** 2)
    sweep_tf = f_sweep / (ms * 1e-3) / 1e12
    roofline = {"bound": "tensor", "kernel": f"k_{dom_name}", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": (achieved / peak) if (achieved and peak) else None, "traffic": traffic,
                "traffic_source": "ncu dram__bytes_read+write of one k_interval launch of 16 chains, scaled by chains",
                "sweep_dense_equivalent": {"tflops": sweep_tf, "frac": (sweep_tf / peak) if peak else None,
                                           "convention": "F = nt*6N^3 + 2N^2*accepted + n_stab*33N^3 per chain-sweep"},
                "peak_source": "measured cuBLAS DGEMM 8192^3 FP64 on this GPU (FP64 has no entry in MEASURED_PEAKS.json)",
                "launch_ms_avg": avg_launch_ms, "launches": int(cnt_cls[dom]),
                "device_ms_by_class": {nm: round(float(v), 3) for nm, v in zip(hq.capi.PROFILE_CLASSES, ms_cls)},
                "launches_by_class": {nm: int(v) for nm, v in zip(hq.capi.PROFILE_CLASSES, cnt_cls)}}
    gpu_launches = int(cnt_cls.sum())
    eng.profile_enable(False)

    # ---- end to end through the C ABI from pinned host buffers ----
    nbytes = n * CFG["nt"] * CFG["nl"] ** 2
    e2e_value = None
    host_fields = torch.empty(nbytes, dtype=torch.int8, pin_memory=True)
    eng.download_fields_i8(host_fields.data_ptr())
    eng.sync()
    host_est = np.zeros((n, 6))
    e2e_steps = 0 if args.no_e2e else max(2, min(args.steps, 6))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        eng.upload_fields_i8(host_fields.data_ptr())  # h2d: this step's field configuration
        eng.init()                                     # stacks + G from the fields
        eng.sweep(hq.SWEEP_UP, hq.SWEEP_MEASURE)
        eng.download_fields_i8(host_fields.data_ptr())  # d2h: updated fields
        host_est = eng.estimators_all()                 # d2h: every chain's estimator sums (synchronises)
    eng.sync()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    if e2e_steps:
        e2e_value = world * n * e2e_steps / e2e_s

    # ---- the plain single-chain GPU path (the 20x bar's denominator) ----
    single = None
    if rank == 0 and not args.no_single:
        one = hq.Engine(chain_params(rank, 1), device=local)
        one.fields_random()
        one.init()
        dd = hq.SWEEP_UP
        for _ in range(2):
            one.sweep(dd)
            dd = hq.SWEEP_DOWN if dd == hq.SWEEP_UP else hq.SWEEP_UP
        one.capture_graph(hq.SWEEP_UP, hq.SWEEP_MEASURE)
        one.capture_graph(hq.SWEEP_DOWN, hq.SWEEP_MEASURE)
        s1 = torch.cuda.ExternalStream(one.stream())
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        one.sync()
        f0.record(s1)
        k1 = 6
        for _ in range(k1):
            one.sweep(dd, hq.SWEEP_MEASURE)
            dd = hq.SWEEP_DOWN if dd == hq.SWEEP_UP else hq.SWEEP_UP
        f1.record(s1)
        torch.cuda.synchronize()
        single = k1 / (f0.elapsed_time(f1) * 1e-3)
        one.close()

    # ---- CPU baseline (rank 0 at N = 1 only, bounded sample) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        procs = os.cpu_count() or 1
        thr, total, wall = cpu_throughput(procs, 1, 0, args.cpu_budget)
        cpu = {"value": thr, "unit": "sweeps/s", "cores": procs, "kind": "port",
               "sample": f"{procs} single-threaded processes, one 12x12 beta=10 chain each, "
                         f"{total} directional sweeps in {wall:.1f} s (OpenBLAS 1 thread each)"}
    eng.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "sweeps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Ising fields, minstd_rand0 seeds 1000+c)",
            "config": {"workload": "DQMC directional update sweeps (wrap + Metropolis + stabilisation + equal-time "
                                   "estimators), 12x12 lattice, beta=10, dt=0.1, nt=100, pace 10",
                       "chains_per_gpu": n, **CFG, "expk_mode": "separable" if expk_mode == 1 else "dense",
                       "delay_depth": kmax, "cuda_graph": True,
                       "autotune": [{"expk": "separable" if t["expk_mode"] == 1 else "dense", "k": t["delay_depth"],
                                     "ms_per_sweep": round(t["ms_per_sweep"], 3), "chosen": t["chosen"]}
                                    for t in tune],
                       "l2": "working set per GPU ~1.8 GB of chain state (> 126 MB L2)"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": ({"value": e2e_value, "unit": "sweeps/s", "h2d_bytes_per_step": nbytes,
                     "d2h_bytes_per_step": nbytes + n * 16 * 8,
                     "step": "h2d fields -> hq_init_stacks_and_g -> hq_sweep(up) -> d2h fields + estimators"}
                    if e2e_value else None),
            "gpu_launches": gpu_launches,
            "clocks": clk,
            "single_chain_gpu": {"value": single, "unit": "sweeps/s",
                                 "batched_over_single": (value / world / single) if single else None},
            "acceptance": accepted / proposed if proposed else None,
            "max_wrap_error": wrap,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of the CPU baseline sample")
    ap.add_argument("--chains", type=int, default=N_CHAINS, help="chains per GPU (256 is the metric's)")
    ap.add_argument("--no-peak", action="store_true", help="skip the DGEMM peak probe")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-single", action="store_true", help="skip the single-chain leg")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (largest delay depth, separable expK)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
