"""torch.autograd.Function over the GPU adjoint of log|det(1 + B(nt-1)...B(0))| (a test
wrapper: every call builds a one-chain engine).

    ld = LogDet.apply(hop, mu, u, fields, beta, pace)

hop: (N, N) symmetric hopping matrix (K = -hop - mu 1, the reference's sign convention of
src/hubbard.cpp:40-41 with t folded into hop), mu and u: 0-d tensors, fields: (nt, N) +-1
array. Forward and backward both come from hq_logdet_adjoint: d/dhop = -dK, d/dmu as
returned, d/du = d/dalpha * dalpha/du with alpha = acosh(exp(dt u / 2)) (src/hubbard.cpp:35).
"""
import math

import numpy as np
import torch

from .capi import Engine


class LogDet(torch.autograd.Function):
    @staticmethod
    def forward(ctx, hop, mu, u, fields, beta, pace):
        fields = np.asarray(fields)
        nt, N = fields.shape
        L = int(round(math.sqrt(N)))
        if L * L != N or tuple(hop.shape) != (N, N):
            raise ValueError("hop must be N x N with N = L^2 = fields.shape[1]")
        muf, uf = float(mu), float(u)
        e = Engine([dict(nl=L, u=uf, mu=muf, beta=float(beta), nt=nt, stabilization_pace=int(pace),
                         expk_mode=0, seed=0)])
        try:
            e.set_hopping(0, hop.detach().to("cpu", torch.float64).numpy())
            e.set_fields(0, fields)
            e.init()
            ld, grads = e.logdet_adjoint()
        finally:
            e.close()
        dmu, dalpha, dK = grads[0]
        dt = float(beta) / nt
        dalpha_du = 0.5 * dt * math.exp(0.5 * dt * uf) / math.sqrt(math.exp(dt * uf) - 1.0)
        ctx.save_for_backward(torch.as_tensor(-dK, dtype=hop.dtype, device=hop.device),
                              torch.as_tensor(dmu, dtype=hop.dtype, device=hop.device),
                              torch.as_tensor(dalpha * dalpha_du, dtype=hop.dtype, device=hop.device))
        return torch.as_tensor(ld[0], dtype=hop.dtype, device=hop.device)

    @staticmethod
    def backward(ctx, g):
        g_hop, g_mu, g_u = ctx.saved_tensors
        return g * g_hop, g * g_mu, g * g_u, None, None, None
