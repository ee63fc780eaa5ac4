"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/dqmc_oracle.cpp into oracle/liboracle.so, linked against the
OpenBLAS that ships inside scipy (the image has no system LAPACK). The product
never loads this library; tests/, smoke() and bench.py's CPU legs do.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "dqmc_oracle.cpp")
OUT = os.path.join(HERE, "liboracle.so")


def openblas_path():
    import scipy
    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    libs = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
    if not libs:
        raise RuntimeError(f"scipy's bundled OpenBLAS not found under {libdir}")
    return libs[0]


def build(force=False):
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    blas = openblas_path()
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC",
           "-o", OUT, SRC, blas, "-Wl,-rpath," + os.path.dirname(blas)]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
