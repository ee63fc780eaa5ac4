"""The C++ facade (include/hubbard_b200.hpp): a driver written against the reference's
DQMC::Core / Model::HubbardAttractiveU surface compiles and links on CPU, and on the GPU
follows the oracle chain of the same seed."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hubbard-attractive-u_b200")


def build_driver(tmp_path):
    exe = str(tmp_path / "shim_driver")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp",
           "shim_driver.cpp"), "-L", PKG, "-lhubbard_b200", "-Wl,-rpath," + PKG, "-o", exe]
    subprocess.check_call(cmd)
    return exe


def test_facade_compiles_and_links(tmp_path):
    exe = build_driver(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_facade_driver_matches_oracle(tmp_path, oracle):
    exe = build_driver(tmp_path)
    out = subprocess.check_output([exe, "42"], text=True).split()
    g00, g11, wrap, fsum = float(out[0]), float(out[1]), float(out[2]), int(out[3])
    o = oracle.OracleChain(4, u=4.0, mu=0.0, beta=4.0, nt=40, pace=10, seed=42)
    o.fields_random()
    o.init()
    for _ in range(2):
        o.sweep(oracle.UP)
        o.sweep(oracle.DOWN)
    g = o.g()
    assert abs(g00 - g[0, 0]) <= 1e-10 and abs(g11 - g[1, 1]) <= 1e-10
    assert fsum == int(o.fields().sum())
    assert 0.0 <= wrap < 1e-8
    # Utils::SvdStack view: left empty, right holding the 4 intervals, positive scales
    assert (int(out[4]), int(out[5]), int(out[6])) == (0, 4, 16) and float(out[7]) > 0.0
