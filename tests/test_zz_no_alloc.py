"""The entry point that allocates no device memory (hq_equaltime_g_noalloc).

It serves callers that cannot call cudaMalloc: a process that hands out its whole
device-memory budget once at start-up, or a service that must never meet an out-of-memory
failure mid-run. Its G(0,0) must equal, within the 1e-10 of the other parity tests, both the
one the allocating path builds (hq_create + hq_set_fields + hq_init_stacks_and_g + hq_get_g)
and the FP64 CPU oracle's, on the same fields, on two calls in a row (the scratch array keeps
the previous call's contents). This file sorts last so that a run stopping at its first
failure has run the rest."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _allocating_path(hq, cfg, fields):
    e = hq.Engine([dict(cfg, seed=1, expk_mode=1)])
    e.set_fields(0, fields)
    e.init()
    g = e.g(0)
    e.close()
    return g


def test_noalloc_matches_allocating_path_and_oracle(hq, oracle):
    import torch
    lib = hq.lib()
    cfg = dict(nl=8, nnt=1.0, u=4.0, mu=-0.5, beta=8.0, nt=160, stabilization_pace=10)
    N = cfg["nl"] ** 2
    stream = torch.cuda.current_stream()
    for seed in (7, 8):  # two calls in a row share the scratch array
        o = oracle.OracleChain(cfg["nl"], nnt=cfg["nnt"], u=cfg["u"], mu=cfg["mu"], beta=cfg["beta"], nt=cfg["nt"],
                               pace=cfg["stabilization_pace"], seed=seed)
        o.fields_random()
        o.init()
        fields = o.fields()
        f_dev = torch.tensor(fields.astype(np.int8), device="cuda")
        g_dev = torch.full((N, N), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.hq_equaltime_g_noalloc(cfg["nl"], cfg["nnt"], cfg["u"], cfg["mu"], cfg["beta"], cfg["nt"],
                                        cfg["stabilization_pace"], f_dev.data_ptr(), g_dev.data_ptr(),
                                        stream.cuda_stream)
        assert rc == 0, hq.capi.last_error()
        torch.cuda.synchronize()
        g_noalloc = g_dev.cpu().numpy().T  # the output is column-major
        g_ref = _allocating_path(hq, cfg, fields)
        assert np.abs(g_noalloc - g_ref).max() <= 1e-10
        assert np.abs(g_noalloc - o.g()).max() <= 1e-10


def test_noalloc_rejects_sizes_beyond_the_scratch(hq):
    import torch
    lib = hq.lib()
    f = torch.ones(100 * 144, dtype=torch.int8, device="cuda")
    g = torch.zeros(144 * 144, dtype=torch.float64, device="cuda")
    rc = lib.hq_equaltime_g_noalloc(12, 1.0, 4.0, 0.0, 10.0, 100, 10, f.data_ptr(), g.data_ptr(), None)
    assert rc == hq.capi.HQ_E_RANGE
    assert "64 sites" in hq.capi.last_error()
