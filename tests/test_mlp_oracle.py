"""The FP64 oracle of the learned pair correction (oracle/mlp_oracle.c), which has no
reference counterpart: checked against an independent PyTorch FP64 autograd restatement of
the MLP (node values, r-derivatives and the parameter backpropagation), against the exact
MLP between nodes (the Hermite tabulation error), and through central differences of the
water oracle with the term switched on (F = -dU/dx, the VJP, sum acoef . dF/dtheta for
classical and MLP parameters, and the reverse-pass gradient)."""

import math

import numpy as np
import pytest

from oracle import orc
from revsim import constants as C, systems

torch = pytest.importorskip("torch")

RC = 1.0


def _torch_u(theta, r):
    """u_tau(r) for all three types at distances r (torch FP64), differentiable in both."""
    H, NR = orc.MLP_H, orc.MLP_NRBF
    mu = torch.arange(NR, dtype=torch.float64) * (RC / (NR - 1))
    w = 0.05
    phi = torch.exp(-(r[:, None] - mu[None, :]) ** 2 / (2 * w * w))
    fc = 0.5 * (torch.cos(math.pi * r / RC) + 1.0)
    out = []
    for t in range(3):
        p = theta[t * orc.MLP_PER_TYPE:(t + 1) * orc.MLP_PER_TYPE]
        W1 = p[:H * NR].reshape(H, NR)
        b1 = p[H * NR:H * NR + H]
        o = H * NR + H
        W2 = p[o:o + H * H].reshape(H, H)
        b2 = p[o + H * H:o + H * H + H]
        w3 = p[o + H * H + H:o + H * H + 2 * H]
        b3 = p[-1]
        h1 = torch.nn.functional.silu(phi @ W1.T + b1)
        h2 = torch.nn.functional.silu(h1 @ W2.T + b2)
        out.append((h2 @ w3 + b3) * fc)
    return torch.stack(out)


@pytest.fixture(scope="module")
def theta():
    th = orc.mlp_init(3)
    th += np.random.default_rng(4).normal(scale=0.05, size=th.shape)   # nonzero biases, larger w3
    return th


def test_nodes_match_torch_autograd(theta):
    u, du = orc.mlp_nodes(theta)
    r = torch.linspace(0, RC, orc.MLP_NG + 1, dtype=torch.float64, requires_grad=True)
    ut = _torch_u(torch.tensor(theta), r)
    assert np.allclose(u, ut.detach().numpy(), rtol=1e-12, atol=1e-12)
    for t in range(3):   # u_tau(r_g) depends on r_g only, so the gradient of the sum is u'
        d = torch.autograd.grad(ut[t].sum(), r, retain_graph=True)[0].numpy()
        assert np.allclose(du[t], d, rtol=1e-10, atol=1e-10)


def test_hermite_table_reproduces_the_mlp_between_nodes(theta):
    coef = orc.mlp_table(theta)
    r = np.linspace(0.1, 0.999, 997) + 0.37 / orc.MLP_NG
    ut = _torch_u(torch.tensor(theta), torch.tensor(r)).numpy()
    scale = np.abs(ut).max()
    for t in range(3):
        ui = np.array([orc.mlp_pair(coef, t, x)[0] for x in r])
        assert np.abs(ui - ut[t]).max() <= 1e-8 * scale


def test_backprop_matches_torch_autograd(theta):
    rng = np.random.default_rng(5)
    adj = rng.normal(size=(3, orc.MLP_NG, 4))
    g = orc.mlp_backprop(theta, adj)
    th = torch.tensor(theta, requires_grad=True)
    r = torch.linspace(0, RC, orc.MLP_NG + 1, dtype=torch.float64, requires_grad=True)
    u = _torch_u(th, r)
    du = torch.stack([torch.autograd.grad(u[t].sum(), r, create_graph=True)[0] for t in range(3)])
    h = RC / orc.MLP_NG
    y0, y1, d0, d1 = u[:, :-1], u[:, 1:], du[:, :-1], du[:, 1:]
    c = torch.stack([y0, h * d0, 3 * (y1 - y0) - h * (2 * d0 + d1), 2 * (y0 - y1) + h * (d0 + d1)], -1)
    (c * torch.tensor(adj)).sum().backward()
    ref = th.grad.numpy()
    assert np.linalg.norm(g - ref) <= 1e-10 * np.linalg.norm(ref)


def _mlp_system(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box, "lj", mlp=True)
    return s, n_mol, box, x, v


def test_forces_with_mlp_are_minus_energy_gradient(small_water, theta):
    s, n_mol, box, x, _ = _mlp_system(small_water)
    p = np.concatenate([C.default_params("lj"), theta])
    pairs = orc.neighbor_pairs(s, x)
    F = orc.forces(s, p, x, pairs)
    F0 = orc.forces(orc.make_system(n_mol, box, "lj"), p[:7], x, pairs)
    assert np.linalg.norm(F - F0) > 1e-3 * np.linalg.norm(F0)   # the term is on
    u = np.random.default_rng(1).normal(size=x.shape)
    h = 1e-7
    dE = (orc.energy(s, p, x + h * u, pairs) - orc.energy(s, p, x - h * u, pairs)) / (2 * h)
    assert abs((F * u).sum() + dE) <= 1e-6 * abs(dE)


def test_vjp_with_mlp_matches_central_difference(small_water, theta):
    s, n_mol, box, x, _ = _mlp_system(small_water)
    p = np.concatenate([C.default_params("lj"), theta])
    pairs = orc.neighbor_pairs(s, x)
    rng = np.random.default_rng(2)
    w = rng.normal(size=x.shape)
    u = rng.normal(size=x.shape)
    _, G, _ = orc.forces_grads(s, p, x, pairs, w, jac=False)
    m = systems.masses(n_mol)[:, None]
    h = 1e-6
    fd = ((w / m) * (orc.forces(s, p, x + h * u, pairs) - orc.forces(s, p, x - h * u, pairs))).sum() / (2 * h)
    assert abs((G * u).sum() - fd) <= 1e-6 * abs(fd)


def test_parameter_contraction_matches_central_difference(small_water, theta):
    s, n_mol, box, x, _ = _mlp_system(small_water)
    p = np.concatenate([C.default_params("lj"), theta])
    pairs = orc.neighbor_pairs(s, x)
    ac = np.random.default_rng(3).normal(size=x.shape)
    g = orc.contract(s, p, x, pairs, ac)
    assert g.shape == (7 + orc.MLP_NPARAMS,)
    Pc = 7
    picks = [0, 2, Pc + 5, Pc + 16 * 64 + 3, Pc + 1088 + 77, Pc + 5248 + 10, Pc + 5312,
             Pc + orc.MLP_PER_TYPE + 900, Pc + 2 * orc.MLP_PER_TYPE + 5300]
    for k in picks:
        hk = 1e-5 * max(abs(p[k]), 1.0)
        pp, pm = p.copy(), p.copy()
        pp[k] += hk
        pm[k] -= hk
        fd = (ac * (orc.forces(s, pp, x, pairs) - orc.forces(s, pm, x, pairs))).sum() / (2 * hk)
        assert abs(g[k] - fd) <= 1e-5 * max(abs(fd), 1e-6 * np.abs(g).max()), (k, g[k], fd)


def test_reverse_gradient_with_mlp_matches_central_difference(small_water, theta):
    s, n_mol, box, x, v = _mlp_system(small_water)
    p = np.concatenate([C.default_params("lj"), theta])
    target = np.linspace(0.5, 1.5, 200)
    loss = orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
    seeds = systems.noise_seeds(20, seed=9)
    xf, vf, lf, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, 20, 20, 0.001, loss, True, 10)
    _, _, lr, g = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, 20, 20, 20, 0.001, sx, sv, loss,
                                  n_steps_log=10)
    assert abs(lr - lf) <= 1e-7 * abs(lf)
    Pc = 7
    for k in [0, Pc + 5, Pc + 1088 + 77, Pc + 5248 + 10, Pc + orc.MLP_PER_TYPE + 5260]:
        hk = 1e-5 * max(abs(p[k]), 1.0)
        pp, pm = p.copy(), p.copy()
        pp[k] += hk
        pm[k] -= hk
        lp = orc.forward_sim(s, pp, x, v, seeds, 1.0, 20, 20, 0.001, loss, True, 10)[2]
        lm = orc.forward_sim(s, pm, x, v, seeds, 1.0, 20, 20, 0.001, loss, True, 10)[2]
        fd = (lp - lm) / (2 * hk)
        assert abs(g[k] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(g).max()), (k, g[k], fd)
