import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels through the C ABI")
    config.addinivalue_line("markers", "slow: long CPU statistics run")


@pytest.fixture(scope="session")
def hq():
    from __graft_entry__ import load_package
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    from oracle import build
    build.build()
    from oracle import oracle as orc
    return orc


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(GOLDEN, "example_run.json")) as f:
        return json.load(f)


def example_fields():
    import numpy as np
    with open(os.path.join(GOLDEN, "example_fields.txt")) as f:
        nt, ns = (int(x) for x in f.readline().split())
        rows = [list(map(int, ln.split())) for ln in f if ln.strip()]
    a = np.array(rows, dtype=np.int32)
    assert a.shape == (nt, ns)
    return a
