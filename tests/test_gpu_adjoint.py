"""GPU tests of the log-det adjoint (no counterpart in the reference) against the oracle's
exact gradient identities and central finite differences (h = 1e-5)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def nn_hop(L):
    N = L * L
    H = np.zeros((N, N))
    for s in range(N):
        x, y = s % L, s // L
        for t in ((x + 1) % L + L * y, x + L * ((y + 1) % L)):
            H[s, t] += 1.0
            H[t, s] += 1.0
    return H


def stream_fields(oracle, L, nt, seed, n):
    """n successive nt x N blocks of one seeded stream (config j = j-th block)."""
    o = oracle.OracleChain(L, nt=nt, beta=1.0, seed=seed)
    out = []
    for _ in range(n):
        o.fields_random()
        out.append(o.fields())
    return out


def test_logdet_gradient_small(hq, oracle):
    L, beta, nt, mu, u = 4, 2.0, 20, -0.3, 4.0
    hop = nn_hop(L)
    fields = stream_fields(oracle, L, nt, 99, 3)
    cfg = dict(nl=L, u=u, mu=mu, beta=beta, nt=nt, stabilization_pace=10, expk_mode=0)
    e = hq.Engine([dict(cfg, seed=c) for c in range(3)])
    for c in range(3):
        e.set_hopping(c, hop)
        e.set_fields(c, fields[c])
    e.init()
    ld, grads = e.logdet_adjoint()
    dt = beta / nt
    for c in range(3):
        o = oracle.OracleChain(L, u=u, mu=mu, beta=beta, nt=nt, pace=10, seed=1, custom_hop=hop)
        o.set_fields(fields[c])
        o.init()
        dmu, dal, dK = o.logdet_grad()
        assert abs(ld[c] - o.logdet()) <= 1e-9 * max(1.0, abs(ld[c]))
        g_mu, g_al, g_K = grads[c]
        assert abs(g_mu - dmu) <= 1e-8 * max(1.0, abs(dmu))
        assert abs(g_al - dal) <= 1e-8 * max(1.0, abs(dal))
        assert np.abs(g_K - dK).max() <= 1e-8 * max(1.0, np.abs(dK).max())

        def logdet(mu_=mu, u_=u, hop_=hop):
            q = oracle.OracleChain(L, u=u_, mu=mu_, beta=beta, nt=nt, pace=10, seed=1, custom_hop=hop_)
            q.set_fields(fields[c])
            return q.logdet()

        h = 1e-5
        fd_mu = (logdet(mu_=mu + h) - logdet(mu_=mu - h)) / (2 * h)
        assert abs(g_mu - fd_mu) <= 1e-6 * max(1.0, abs(fd_mu))
        # alpha enters through u: alpha = acosh(exp(dt u / 2))
        dalpha_du = 0.5 * dt * math.exp(0.5 * dt * u) / math.sqrt(math.exp(dt * u) - 1.0)
        fd_u = (logdet(u_=u + h) - logdet(u_=u - h)) / (2 * h)
        assert abs(g_al * dalpha_du - fd_u) <= 1e-6 * max(1.0, abs(fd_u))
        # per-bond hopping t_b on (i, j): K_ij = K_ji = -t_b  =>  d/dt_b = -(Gamma_ij + Gamma_ji)
        for (i, j) in ((0, 1), (5, 9), (15, 3)):
            if hop[i, j] == 0:
                continue
            hp, hm = hop.copy(), hop.copy()
            hp[i, j] += h; hp[j, i] += h
            hm[i, j] -= h; hm[j, i] -= h
            fd_b = (logdet(hop_=hp) - logdet(hop_=hm)) / (2 * h)
            g_b = -(g_K[i, j] + g_K[j, i])
            assert abs(g_b - fd_b) <= 1e-6 * max(1.0, abs(fd_b)), (i, j, g_b, fd_b)
    e.close()


def test_density_identity(hq, oracle):
    """d logdet / d mu = dt sum_l tr(1 - G_l) = beta N n / 2 with n the reference's filling
    estimator of the same fields (include/observable_methods.hpp:39-52)."""
    L, beta, nt = 4, 2.0, 20
    fields = stream_fields(oracle, L, nt, 5, 1)[0]
    e = hq.Engine([dict(nl=L, u=4.0, mu=-0.3, beta=beta, nt=nt, stabilization_pace=10, seed=1, expk_mode=0)])
    e.set_fields(0, fields)
    e.init()
    _, grads = e.logdet_adjoint()
    o = oracle.OracleChain(L, u=4.0, mu=-0.3, beta=beta, nt=nt, pace=10, seed=1, equaltime=True, dynamic=True)
    o.set_fields(fields)
    o.init()
    o.sweep(oracle.DYNAMIC)  # no-update pass: vecgftt of the fixed fields
    n = o.measure_equaltime()[0]
    assert abs(grads[0][0] - beta * L * L * n / 2) <= 1e-9 * abs(grads[0][0])
    e.close()


def test_c4_batched_configurations(hq, oracle):
    """10x10, mu=-0.3, U=-4, beta=6, dt=0.1, pace 10, 64 configurations of seed 99: all
    gradients in one batched call; two of them checked against central differences."""
    L, beta, nt, mu, u = 10, 6.0, 60, -0.3, 4.0
    hop = nn_hop(L)
    fields = stream_fields(oracle, L, nt, 99, 64)
    e = hq.Engine([dict(nl=L, u=u, mu=mu, beta=beta, nt=nt, stabilization_pace=10, seed=c, expk_mode=0)
                   for c in range(64)])
    for c in range(64):
        e.set_hopping(c, hop)
        e.set_fields(c, fields[c])
    e.init()
    ld, grads = e.logdet_adjoint()
    assert np.all(np.isfinite(ld))
    h = 1e-5
    for c in (0, 63):
        def logdet(mu_=mu, hop_=hop):
            q = oracle.OracleChain(L, u=u, mu=mu_, beta=beta, nt=nt, pace=10, seed=1, custom_hop=hop_)
            q.set_fields(fields[c])
            return q.logdet()
        fd_mu = (logdet(mu_=mu + h) - logdet(mu_=mu - h)) / (2 * h)
        assert abs(grads[c][0] - fd_mu) <= 1e-6 * abs(fd_mu)
        i, j = 0, 1
        hp, hm = hop.copy(), hop.copy()
        hp[i, j] += h; hp[j, i] += h
        hm[i, j] -= h; hm[j, i] -= h
        fd_b = (logdet(hop_=hp) - logdet(hop_=hm)) / (2 * h)
        g_b = -(grads[c][2][i, j] + grads[c][2][j, i])
        assert abs(g_b - fd_b) <= 1e-6 * max(1.0, abs(fd_b))
    e.close()


def test_autograd_function_gradcheck(hq, oracle):
    """The torch.autograd.Function wrapper: gradients with respect to the 2N bond hoppings,
    mu and u against torch's own central differences of the GPU log-determinant."""
    import torch
    from hubbard_b200.autograd import LogDet

    L, beta, nt, pace = 3, 1.0, 10, 5
    N = L * L
    H = nn_hop(L)
    bonds = [(i, j) for i in range(N) for j in range(i + 1, N) if H[i, j] != 0]
    fields = stream_fields(oracle, L, nt, 99, 1)[0]
    rng = np.random.default_rng(5)
    t = torch.tensor(1.0 + 0.1 * rng.standard_normal(len(bonds)), dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(-0.3, dtype=torch.float64, requires_grad=True)
    u = torch.tensor(4.0, dtype=torch.float64, requires_grad=True)
    ii = torch.tensor([b[0] for b in bonds])
    jj = torch.tensor([b[1] for b in bonds])

    def f(t_, mu_, u_):
        hop = torch.zeros(N, N, dtype=torch.float64)
        hop = hop.index_put((ii, jj), t_, accumulate=True).index_put((jj, ii), t_, accumulate=True)
        return LogDet.apply(hop, mu_, u_, fields, beta, pace)

    assert torch.autograd.gradcheck(f, (t, mu, u), eps=1e-5, atol=1e-5, rtol=1e-4)
    # the value is the oracle's log-determinant of the same hopping matrix
    hop = np.zeros((N, N))
    tv = t.detach().numpy()
    for k, (i, j) in enumerate(bonds):
        hop[i, j] += tv[k]
        hop[j, i] += tv[k]
    o = oracle.OracleChain(L, u=4.0, mu=-0.3, beta=beta, nt=nt, pace=pace, seed=1, custom_hop=hop)
    o.set_fields(fields)
    ld = float(f(t, mu, u).detach())
    assert abs(ld - o.logdet()) <= 1e-9 * max(1.0, abs(ld))
