#!/usr/bin/env python
"""Throughput of the batched DQMC sweep on B200.

Default workload (the metric's configuration): 256 independent Markov chains of the
attractive-U Hubbard model on a 12x12 periodic lattice (N = 144), t = 1, |U| = 4, mu = 0,
beta = 10, dt = 0.1 (nt = 100 slices), stabilisation every 10 slices, Ising fields i.i.d. +-1
from per-chain seeds 1000 + c (the reference's minstd_rand0 stream), thermalised by 200
directional sweeps before timing. One step = one directional update sweep (the reference's
unit, src/dqmc_handle.cpp:72) of every chain, alternating 0 -> beta and beta -> 0, with the
fused equal-time estimators on.

  value : aggregate directional sweeps/s with the chains resident in HBM (CUDA events
          on the library's stream around K captured-graph sweeps, max over ranks)
  e2e   : the same metric through the C ABI from host buffers. One step is one round trip,
          the unit of the reference's measurement loop (src/dqmc_handle.cpp:145-150): the
          fields are copied host -> device, the stacks and G are built from them
          (hq_init_stacks_and_g), an up and a down sweep run with the estimators on, and
          fields + estimator sums are copied back; two directional sweeps per step.
  g_err_vs_oracle : after the timed steps, the freshly stabilised G of chain 0 against the
          FP64 CPU oracle's G(0,0) from the same fields (pace 1 and pace 10), outside the
          timed region.
  --impl reference : the CPU restatement of the reference path (oracle/) on all host
          cores, one chain per process, same configuration and unit.
  --workload c3 | c5 : the batched uneven configuration (256 chains, L in {6..12}, |U| in
          {2,4,6}, beta in {4,8,12}) or the large one (64 chains of 16x16, beta = 16,
          nt = 320, pace 8), timed the same way (value only).

Multi-GPU (torchrun): every rank runs its own chains (weak scaling, no collective in the data
path); the elapsed time is the max over ranks.
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
EXAMPLE = dict(nl=4, nnt=1.0, u=4.0, mu=0.0, beta=8.0, nt=160, stabilization_pace=10)  # example/config.toml


def chain_params(rank, n=N_CHAINS, expk_mode=-1):
    """The metric's chains: seeds 1000 + c, c counted across ranks."""
    return [dict(CFG, seed=SEED0 + rank * n + c, expk_mode=expk_mode) for c in range(n)]


def c3_params(rank, n=256):
    """Batched uneven chains: L = 6, 8, 10, 12 (a quarter each), |U| = 2, 4, 6 and
    beta = 4, 8, 12 cycled (dt = 0.1), pace 10, seeds 1000 + c."""
    out = []
    for c in range(n):
        beta = [4.0, 8.0, 12.0][(c // 3) % 3]
        out.append(dict(nl=[6, 8, 10, 12][(c * 4) // n], nnt=1.0, u=[2.0, 4.0, 6.0][c % 3], mu=0.0, beta=beta,
                        nt=int(round(beta / 0.1)), stabilization_pace=10, seed=SEED0 + rank * n + c, expk_mode=-1))
    return out


def c5_params(rank, n=64):
    """Large batched run: 16x16, mu = -0.2, beta = 16, dt = 0.05 (nt = 320), pace 8, seeds 5000 + c."""
    return [dict(nl=16, nnt=1.0, u=4.0, mu=-0.2, beta=16.0, nt=320, stabilization_pace=8, seed=5000 + rank * n + c,
                 expk_mode=-1) for c in range(n)]


WORKLOADS = {
    "metric": ("DQMC directional update sweeps (wrap + Metropolis + stabilisation + equal-time estimators), "
               "12x12 lattice, beta=10, dt=0.1, nt=100, pace 10", chain_params, N_CHAINS),
    "c3": ("DQMC directional update sweeps of 256 uneven chains: L in {6,8,10,12} (64 each), |U| in {2,4,6} "
           "and beta in {4,8,12} cycled, dt=0.1, pace 10", c3_params, 256),
    "c5": ("DQMC directional update sweeps of 64 chains of 16x16, mu=-0.2, beta=16, dt=0.05, nt=320, pace 8",
           c5_params, 64),
}


# --------------------------------------------------------------------------------------
#  CPU legs (the oracle is the checker and the timed CPU baseline only)
# --------------------------------------------------------------------------------------
def _cpu_worker(args):
    seed, warm, steps, budget_s, cfg, threads = args
    from oracle.oracle import OracleChain, set_num_threads, UP, DOWN
    set_num_threads(threads)
    ch = OracleChain(cfg["nl"], nnt=cfg["nnt"], u=cfg["u"], mu=cfg["mu"], beta=cfg["beta"], nt=cfg["nt"],
                     pace=cfg["stabilization_pace"], seed=seed)
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


def cpu_throughput(procs, warm, steps, budget_s, cfg=CFG, threads=1):
    """Aggregate directional sweeps/s of `procs` oracle chains with `threads` BLAS threads each."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(SEED0 + p, warm, steps, budget_s, cfg, threads) for p in range(procs)])
    total = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    return total / wall, total, wall


def cpu_baseline_leg(budget_s):
    """The oracle on the host cores: P single-threaded chains (the MPI-rank analogue, the
    baseline), one chain with P BLAS threads, and the reference's example configuration
    (L=4, beta=8, nt=160) per core for comparison with its published ~253 sweeps/s/rank."""
    procs = os.cpu_count() or 1
    thr, total, wall = cpu_throughput(procs, 1, 0, budget_s)
    thr_t, total_t, wall_t = cpu_throughput(1, 1, 0, max(3.0, budget_s / 3), threads=procs)
    thr_e, total_e, wall_e = cpu_throughput(procs, 2, 0, max(3.0, budget_s / 3), cfg=EXAMPLE)
    return {"value": thr, "unit": "sweeps/s", "cores": procs, "kind": "port",
            "sample": f"{procs} single-threaded processes, one 12x12 beta=10 chain each, "
                      f"{total} directional sweeps in {wall:.1f} s (OpenBLAS 1 thread each)",
            "threaded_blas": {"value": thr_t, "unit": "sweeps/s", "threads": procs,
                              "sample": f"1 process, OpenBLAS {procs} threads, {total_t} sweeps in {wall_t:.1f} s"},
            "example_config": {"value_per_core": thr_e / procs, "unit": "sweeps/s per core",
                               "published_per_rank": 253.3, "published_source": "example/log.out:40 of the reference",
                               "sample": f"{procs} processes, L=4 beta=8 nt=160 pace 10, {total_e} sweeps in "
                                         f"{wall_e:.1f} s"}}


def oracle_g_check(G_gpu, fields, cfg):
    """Max-abs difference between the GPU's freshly stabilised G and the oracle's G(0,0) of
    the same fields, stabilised every slice (pace 1) and as configured (pace 10)."""
    import numpy as np
    from oracle.oracle import OracleChain, set_num_threads
    set_num_threads(1)
    out = {}
    for pace in (1, cfg["stabilization_pace"]):
        o = OracleChain(cfg["nl"], nnt=cfg["nnt"], u=cfg["u"], mu=cfg["mu"], beta=cfg["beta"], nt=cfg["nt"],
                        pace=pace, seed=0)
        o.set_fields(fields)
        o.init()
        g = o.g()
        out[f"pace{pace}"] = {"max_abs": float(np.abs(G_gpu - g).max()), "max_abs_G": float(np.abs(g).max())}
    p1 = out["pace1"]
    out["rel_to_max_G"] = p1["max_abs"] / max(1.0, p1["max_abs_G"])
    out["chain"] = 0
    return out


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
    """Algorithmic FP64 flops of the interval kernel for one chain: wraps of n_slices slices
    plus `accepted` flips in submatrix form (blocks of kmax sites): per flip the rank-1 share of
    the DMMA flush (2 N^2) and its panel row / column (4 N m for the m-th flip of a block)."""
    N = nl * nl
    wrap = (8.0 * N * nl ** 3) if expk_mode == 1 else (4.0 * N ** 3)  # two expK applications per slice
    blocks = n_slices * ((N + kmax - 1) // kmax)
    per_block = accepted / blocks if blocks else 0.0
    mbar = max(per_block - 1.0, 0.0) / 2.0  # mean in-block index of an accepted flip
    flip = 2.0 * N * N + 4.0 * N * mbar
    return n_slices * wrap + accepted * flip


def sweep_flops(p, sweeps, accepted, kmax, expk_mode):
    """Algorithmic FP64 flops of whole directional sweeps of one chain, as the persistent sweep
    kernel performs them: the interval work (interval_flops) plus, per stabilisation interval,
    the B chain of its slices (4 N L^3 per slice separable, 2 N^3 dense), the UDV factorisation
    with the formation of Q (8/3 N^3), the cumulative V^T (2 N^3), the four builder products
    (8 N^3) and the inverse (2 N^3)."""
    nl, nt = p["nl"], p["nt"]
    N = nl * nl
    n_stab = -(-nt // p["stabilization_pace"])
    bchain = (4.0 * N * nl ** 3) if expk_mode == 1 else (2.0 * N ** 3)
    stab = sweeps * (nt * bchain + n_stab * (8.0 / 3.0 + 2.0 + 8.0 + 2.0) * N ** 3)
    return interval_flops(nl, nt * sweeps, accepted, kmax, expk_mode) + stab


def dense_equivalent_flops(p, sweeps, accepted):
    """One chain's sweeps in the dense-GEMM convention: nt 6N^3 + n_stab 33N^3 per sweep and
    2N^2 per accepted flip."""
    N = p["nl"] ** 2
    n_stab = -(-p["nt"] // p["stabilization_pace"])
    return sweeps * (p["nt"] * 6.0 * N ** 3 + n_stab * 33.0 * N ** 3) + accepted * 2.0 * N ** 2


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
    wl_desc, wl_params, wl_n = WORKLOADS[args.workload]
    metric_wl = args.workload == "metric"
    n = args.chains if args.chains else wl_n
    peak = fp64_peak_tflops(torch, local) if not args.no_peak else None

    params = wl_params(rank, n)
    eng = hq.Engine(params, device=local)
    eng.fields_random()
    eng.init()
    # expK application and delay depth picked by timing (the chains' state is restored)
    tune = [] if args.no_tune else eng.autotune(sweeps=1)
    cfgs = [eng.config(c) for c in range(n)]
    stream = torch.cuda.ExternalStream(eng.stream())
    eng.profile_enable(True)
    eng.capture_graph(hq.SWEEP_UP, hq.SWEEP_MEASURE)
    eng.capture_graph(hq.SWEEP_DOWN, hq.SWEEP_MEASURE)
    # thermalisation (untimed) and W warm-up sweeps, alternating directions
    d = hq.SWEEP_UP
    for _ in range(args.thermalize + max(args.warmup, 3)):
        eng.sweep(d, hq.SWEEP_MEASURE)
        d = hq.SWEEP_DOWN if d == hq.SWEEP_UP else hq.SWEEP_UP
    eng.sync()
    eng.reset_estimators(reset_wrap=True)
    acc0 = eng.estimators_all()

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
    acc1 = eng.estimators_all()
    acc_chain = acc1[:, 5] - acc0[:, 5]
    accepted = float(acc_chain.sum())
    proposed = float((acc1[:, 4] - acc0[:, 4]).sum())
    wrap = max(eng.wrap_errors(c)[0] for c in range(n))
    value = world * n * args.steps / (ms * 1e-3)

    # roofline of the dominant kernel class (largest share of device time)
    dom = int(np.argmax(ms_cls))
    dom_name = hq.capi.PROFILE_CLASSES[dom]
    avg_launch_ms = ms_cls[dom] / max(1, cnt_cls[dom])
    if dom_name in ("interval", "interval_cluster"):
        flops_total = sum(interval_flops(p["nl"], p["nt"] * args.steps, acc_chain[c], cfgs[c][1], cfgs[c][0])
                          for c, p in enumerate(params))
        flops_per_launch = flops_total / max(1, cnt_cls[dom])
    elif dom_name == "sweep":
        flops_total = sum(sweep_flops(p, args.steps, acc_chain[c], cfgs[c][1], cfgs[c][0]) for c, p in enumerate(params))
        flops_per_launch = flops_total / max(1, cnt_cls[dom])
    else:
        flops_per_launch = None
    achieved = (flops_per_launch / (avg_launch_ms * 1e-3) / 1e12) if flops_per_launch else None
    traffic = None
    if dom_name == "interval" and metric_wl:
        # DRAM bytes of one k_interval launch: ncu capture of a 16-chain launch of this workload
        # (2.864 MB read, 0 written: the chains' G and fields), scaled by the chains of one launch
        # here (the traffic is per-chain state; with two chain groups a launch covers half of them)
        chains_per_launch = n * (CFG["nt"] // CFG["stabilization_pace"]) * args.steps / max(1, int(cnt_cls[dom]))
        traffic = 2.864e6 * chains_per_launch / 16
    f_sweep = world * sum(dense_equivalent_flops(p, args.steps, acc_chain[c]) for c, p in enumerate(params))
    sweep_tf = f_sweep / (ms * 1e-3) / 1e12
    sweep_mode = "persistent" if eng.sweep_mode() == hq.SWEEP_PERSISTENT else "launches"
    roofline = {"bound": "tensor", "kernel": f"k_{dom_name}", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": (achieved / peak) if (achieved and peak) else None, "traffic": traffic,
                "traffic_source": ("ncu dram__bytes_read+write of one k_interval launch of 16 chains, scaled by chains"
                                   if traffic else None),
                "flops_convention": ("whole sweep: interval work (separable wrap 8NL^3 per slice, 2N^2 + 4N m per "
                                     "accepted flip) + per interval B chain, UDV 8/3 N^3, V^T 2N^3, builder 8N^3, "
                                     "inverse 2N^3" if dom_name == "sweep" else
                                     "interval work: separable wrap 8NL^3 per slice, 2N^2 + 4N m per accepted flip"),
                "sweep_dense_equivalent": {"tflops": sweep_tf, "frac": (sweep_tf / peak) if peak else None,
                                           "convention": "F = nt*6N^3 + 2N^2*accepted + n_stab*33N^3 per chain-sweep"},
                "peak_source": "measured cuBLAS DGEMM 8192^3 FP64 on this GPU (FP64 has no entry in MEASURED_PEAKS.json)",
                "launch_ms_avg": avg_launch_ms, "launches": int(cnt_cls[dom]),
                "device_ms_by_class": {nm: round(float(v), 3) for nm, v in zip(hq.capi.PROFILE_CLASSES, ms_cls)},
                "launches_by_class": {nm: int(v) for nm, v in zip(hq.capi.PROFILE_CLASSES, cnt_cls)}}
    gpu_launches = int(cnt_cls.sum())
    eng.profile_enable(False)

    # ---- G of chain 0 against the FP64 oracle (outside the timed region) ----
    g_check = None
    if metric_wl and rank == 0 and not args.no_cpu:
        g_check = oracle_g_check(eng.g(0), eng.fields(0), params[0])

    # ---- the dominant kernel alone: 128 of the chains on one stream (no chain groups), outside
    # the timed region; its launches then occupy the GPU alone ----
    isolated = None
    if metric_wl and rank == 0 and dom_name == "interval" and not args.no_isolated:
        ns = min(128, len(params))
        os.environ["HQ_CHAIN_GROUPS"] = "1"
        try:
            solo = hq.Engine(params[:ns], device=local)
        finally:
            os.environ.pop("HQ_CHAIN_GROUPS", None)
        solo.fields_random()
        solo.init()
        sd = hq.SWEEP_UP
        for _ in range(2):
            solo.sweep(sd, hq.SWEEP_MEASURE)
            sd = hq.SWEEP_DOWN if sd == hq.SWEEP_UP else hq.SWEEP_UP
        solo.sync()
        a0 = solo.estimators_all()
        solo.profile_enable(True)
        ms2 = np.zeros(len(hq.capi.PROFILE_CLASSES))
        cnt2 = np.zeros(len(hq.capi.PROFILE_CLASSES), dtype=np.int64)
        for _ in range(2):
            solo.sweep(sd, hq.SWEEP_MEASURE)
            solo.profile_collect(ms2, cnt2)
            sd = hq.SWEEP_DOWN if sd == hq.SWEEP_UP else hq.SWEEP_UP
        a1 = solo.estimators_all()
        ic = hq.capi.PROFILE_CLASSES.index("interval")
        ccfg = [solo.config(c) for c in range(ns)]
        fl = sum(interval_flops(p["nl"], p["nt"] * 2, a1[c, 5] - a0[c, 5], ccfg[c][1], ccfg[c][0])
                 for c, p in enumerate(params[:ns]))
        launch_ms = ms2[ic] / max(1, cnt2[ic])
        ach = fl / max(1, cnt2[ic]) / (launch_ms * 1e-3) / 1e12
        isolated = {"chains_per_launch": ns, "launch_ms_avg": launch_ms, "achieved": ach,
                    "frac": (ach / peak) if peak else None,
                    "note": f"k_interval timed on one stream with no other kernel beside it (a context of {ns} of "
                            "the chains with HQ_CHAIN_GROUPS=1), outside the timed region"}
        solo.close()
    roofline["isolated"] = isolated

    # ---- end to end through the C ABI from pinned host buffers: one round trip per step ----
    e2e = None
    if metric_wl and not args.no_e2e:
        nbytes = sum(p["nt"] * p["nl"] ** 2 for p in params)
        host_fields = torch.empty(nbytes, dtype=torch.int8, pin_memory=True)
        eng.download_fields_i8(host_fields.data_ptr())
        eng.sync()
        e2e_steps = max(2, min(args.steps // 2, 5))
        eng.capture_graph(hq.SWEEP_UP, hq.SWEEP_MEASURE)
        eng.capture_graph(hq.SWEEP_DOWN, hq.SWEEP_MEASURE)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            eng.upload_fields_i8(host_fields.data_ptr())    # h2d: this step's field configurations
            eng.init()                                       # stacks + G from the fields
            eng.sweep(hq.SWEEP_UP, hq.SWEEP_MEASURE)
            eng.sweep(hq.SWEEP_DOWN, hq.SWEEP_MEASURE)
            eng.download_fields_i8(host_fields.data_ptr())  # d2h: updated fields
            eng.estimators_all()                             # d2h: every chain's estimator sums (synchronises)
        eng.sync()
        e2e_s = time.perf_counter() - t0
        if dist:
            t = torch.tensor([e2e_s], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": world * n * 2 * e2e_steps / e2e_s, "unit": "sweeps/s", "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes + n * 6 * 8, "steps": e2e_steps,
               "step": "h2d fields -> hq_init_stacks_and_g -> hq_sweep(up) -> hq_sweep(down) -> d2h fields + "
                       "estimators (two directional sweeps per step)"}

    # ---- the plain single-chain GPU path (the 20x bar's denominator) ----
    single = None
    if metric_wl and rank == 0 and not args.no_single:
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
    if metric_wl and rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_leg(args.cpu_budget)
    eng.close()
    if rank == 0:
        modes = sorted({"separable" if m == 1 else "dense" for m, _ in cfgs})
        depths = sorted({k for _, k in cfgs})
        config = {"workload": wl_desc, "chains_per_gpu": n}
        if metric_wl:
            config.update(CFG)
        config.update({"sweep_mode": sweep_mode, "expk_mode": modes[0] if len(modes) == 1 else modes,
                       "delay_depth": depths[0] if len(depths) == 1 else depths, "cuda_graph": True,
                       "thermalization_sweeps": args.thermalize,
                       "autotune": [{"nl": t["nl"], "expk": {1: "separable", 0: "dense"}.get(t["expk_mode"], "-"),
                                     "k": t["delay_depth"], "cluster": t["cluster_size"],
                                     "sweep": "persistent" if t["sweep_mode"] == hq.SWEEP_PERSISTENT else "launches",
                                     "ms_per_sweep": round(t["ms_per_sweep"], 3), "chosen": t["chosen"]} for t in tune],
                       "l2": "working set per GPU of chain state far above the 126 MB L2 (no flush needed)"})
        line = {
            "metric": METRIC if metric_wl else f"sweeps/s ({args.workload})", "value": value, "unit": "sweeps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Ising fields, minstd_rand0 seeds per chain)",
            "config": config,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": gpu_launches,
            "clocks": clk,
            "single_chain_gpu": ({"value": single, "unit": "sweeps/s",
                                  "batched_over_single": (value / world / single) if single else None}
                                 if metric_wl else None),
            "acceptance": accepted / proposed if proposed else None,
            "max_wrap_error": wrap,
            "g_err_vs_oracle": g_check,
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
    ap.add_argument("--workload", default="metric", choices=sorted(WORKLOADS))
    ap.add_argument("--thermalize", type=int, default=200, help="untimed directional sweeps before the warm-up")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU legs (baseline and oracle G check)")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of the CPU baseline sample")
    ap.add_argument("--chains", type=int, default=0, help="chains per GPU (default: the workload's)")
    ap.add_argument("--no-peak", action="store_true", help="skip the DGEMM peak probe")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-single", action="store_true", help="skip the single-chain leg")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (largest delay depth, separable expK)")
    ap.add_argument("--no-isolated", action="store_true", help="skip the dominant kernel timed alone")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
