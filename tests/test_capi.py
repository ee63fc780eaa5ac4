"""CPU tests of the C ABI library: it loads, exports every declared entry point and
reports errors through return codes (no compute calls without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hubbard_b200.h")


def declared_symbols():
    return re.findall(r"HQ_API\s+int\s+(hq_\w+)\s*\(", open(HEADER).read())


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 20
    assert "hq_sweep" in names and "hq_create" in names and "hq_logdet_adjoint" in names


def test_library_exports_every_declared_symbol(hq):
    lib = hq.lib()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(hq.EXPORTS) == set(declared_symbols())


def test_library_is_sm100a():
    so = os.path.join(ROOT, "hubbard-attractive-u_b200", "libhubbard_b200.so")
    out = subprocess.run(["cuobjdump", "--list-elf", so], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_errors_are_return_codes(hq):
    lib = hq.lib()
    # invalid arguments never abort: a status code and a message
    rc = lib.hq_create(0, 0, None, None)
    assert rc == hq.capi.HQ_E_INVALID
    assert "invalid" in hq.capi.last_error()
    assert lib.hq_sweep(None, 0, 0) == hq.capi.HQ_E_INVALID
    assert lib.hq_get_g(None, 0, 0, 0, None) != 0


def test_parameter_checks_match_reference(hq):
    # include/dqmc_parser.hpp:124-132: u >= 0 (before any device work)
    p = hq.capi.HqChainParams(4, 1.0, -1.0, 0.0, 4.0, 40, 10, 0, 1, 0, 0, 0)
    h = ctypes.c_void_p()
    rc = hq.lib().hq_create(0, 1, ctypes.byref(p), ctypes.byref(h))
    assert rc != 0
