"""Build recipe of the in-tree CUDA library libhubbard_b200.so (sm_100a).

nvcc cross-compiles for sm_100a without a GPU. Every translation unit of csrc/ is compiled to
an object file under _build/ (in parallel, and again only when its source or a header
changed); the objects are linked into the shared library next to this file, so that it
travels with the repository to the GPU host.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libhubbard_b200.so")
SOURCES = ["hq_sweep.cu", "hq_interval.cu", "hq_interval_cluster.cu", "hq_udt.cu", "hq_invert.cu", "hq_gemm.cu",
           "hq_kernels.cu", "hq_engine.cu"]
HEADERS = ["hq_types.h", "hq_device.cuh", "hq_common.cuh", "hq_metropolis.cuh", "hq_kernels.h", "hq_interval.cuh",
           "hq_udt.cuh", "hq_invert.cuh", "hq_phases.cuh", "hq_cta_gemm.cuh"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]


def _headers():
    files = [os.path.join(CSRC, f) for f in HEADERS]
    files.append(os.path.join(os.path.dirname(HERE), "include", "hubbard_b200.h"))
    return files


def _obj(src):
    return os.path.join(BUILD, os.path.splitext(src)[0] + ".o")


def _stale(target, inputs):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(f) > t for f in inputs)


def up_to_date():
    objs = [_obj(s) for s in SOURCES]
    if _stale(OUT, [os.path.join(CSRC, s) for s in SOURCES] + _headers()):
        return False
    return not any(not os.path.exists(o) for o in objs) or os.path.exists(OUT)


def build(force=False, verbose=False, extra_flags=()):
    if not force and not extra_flags and up_to_date():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(BUILD, exist_ok=True)
    jobs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        if force or extra_flags or _stale(_obj(s), [src] + _headers()):
            jobs.append([nvcc, *NVCC_FLAGS, *extra_flags, "-c", "-o", _obj(s), src])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        futs = []
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd), flush=True)
            futs.append(ex.submit(subprocess.run, cmd, capture_output=True, text=True))
        failed = []
        for cmd, f in zip(jobs, futs):
            r = f.result()
            if r.stdout or r.stderr:
                sys.stdout.write(r.stdout + r.stderr)
            if r.returncode != 0:
                failed.append(cmd[-1])
        if failed:
            raise RuntimeError("nvcc failed on " + ", ".join(failed))
    link = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT] + [_obj(s) for s in SOURCES]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.check_call(link)
    return OUT


if __name__ == "__main__":
    flags = [a for a in sys.argv[1:] if a.startswith("-D")]
    print(build(force="--force" in sys.argv, verbose=True, extra_flags=flags))
