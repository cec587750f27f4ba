"""The oracle's learned radial term on the Stillinger-Weber diamond path (one MLP type on
[0, 0.25 nm] added to the 2-body term of every active pair) against independent checks:
the energy difference against a numpy evaluation of the tabulated term over the pair set;
F = -dU/dx, the Hessian-vector product, the parameter contraction, the stress-loss
derivatives and the reverse-pass gradient of the reference's self-check run against central
differences, for the MLP parameters as for the SW ones.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import diamond as D, mlp

P0 = D.default_params()
RC, W = orc.SW_MLP_RC, orc.SW_MLP_WIDTH
# MLP parameters probed by central differences: W1, b1, W2, b2, w3 and b3 entries
PROBES = [3, 1024 + 7, 1088 + 70, 1088 + 4096 + 5, 5248 + 11, 5312]


def _step(theta, k, rel):
    """Central-difference step: relative for the SW parameters; 1e-4 for the MLP ones (the
    forces and losses are ~1e4-1e6 times their MLP derivatives, so smaller steps drown in
    rounding, and they are smooth in the weights)."""
    return rel * abs(theta[k]) if k < 7 else 1e-4


def _rtol(k):
    """1e-6 for the SW parameters; 1e-5 for the MLP ones, whose central differences carry
    ~1e-7 relative rounding (the step is 1e-4 on a sum of ~1e5)."""
    return 1e-6 if k < 7 else 1e-5


def _gmax(g, k):
    """Largest entry of k's group (SW or MLP parameters): the floor of the relative test."""
    return np.abs(g[:7]).max() if k < 7 else np.abs(g[7:]).max()


@pytest.fixture(scope="module")
def crystal():
    x, box = D.diamond_coords(3, noise=0.01, seed=4)
    v = D.mb_velocities(len(x), seed=5)
    return box, x, v


@pytest.fixture(scope="module")
def theta():
    """SW parameters followed by a strongly-on MLP (the seeded initialisation of one type
    perturbed by N(0, 0.1))."""
    th = mlp.init_params(3)[:mlp.PER_TYPE] + np.random.default_rng(8).normal(scale=0.1, size=mlp.PER_TYPE)
    return np.concatenate([P0, th])


def _pairs_r(x, box, p):
    d = x[None, :, :] - x[:, None, :]
    d -= np.round(d / box) * box
    r = np.linalg.norm(d, axis=2)
    i, j = np.nonzero(np.triu(r < p[2] * p[5], 1))
    return r[i, j]


def test_energy_adds_the_tabulated_term(crystal, theta):
    box, x, _ = crystal
    s, s0 = orc.make_sw_system(len(x), box, mlp=True), orc.make_sw_system(len(x), box)
    assert orc.sw_n_params(s) == 7 + mlp.PER_TYPE
    coef = orc.mlp_table_n(theta[7:], 1, RC, W)[0]
    r = _pairs_r(x, box, P0)
    r = r[r < RC]
    h = RC / orc.MLP_NG
    g = np.minimum((r / h).astype(int), orc.MLP_NG - 1)
    sv = r / h - g
    c = coef[g]
    u = c[:, 0] + sv * (c[:, 1] + sv * (c[:, 2] + sv * c[:, 3]))
    dE = orc.sw_energy(s, theta, x) - orc.sw_energy(s0, P0, x)
    assert len(r) > 100 and abs(u.sum()) > 1.0
    assert abs(dE - u.sum()) <= 1e-9 * np.abs(u).sum()


def test_forces_and_hessian_vector_product(crystal, theta):
    box, x, _ = crystal
    s = orc.make_sw_system(len(x), box, mlp=True)
    rng = np.random.default_rng(2)
    u = rng.normal(size=x.shape)
    w = rng.normal(size=x.shape)
    h = 1e-6
    F, G, _ = orc.sw_forces_grads(s, theta, x, w, jac=False)
    dE = (orc.sw_energy(s, theta, x + h * u) - orc.sw_energy(s, theta, x - h * u)) / (2 * h)
    assert abs((F * u).sum() + dE) <= 1e-7 * abs(dE)
    # dl_dfi = J (w / m), J = dF/dx symmetric: u . J (w/m) = d/dh (F(x + h w/m) . u)
    wm = w / s.mass
    fd = ((orc.sw_forces(s, theta, x + h * wm) - orc.sw_forces(s, theta, x - h * wm)) * u).sum() / (2 * h)
    assert abs((G * u).sum() - fd) <= 1e-6 * abs(fd)


def test_parameter_contraction(crystal, theta):
    box, x, _ = crystal
    s = orc.make_sw_system(len(x), box, mlp=True)
    ac = np.random.default_rng(3).normal(size=x.shape)
    th = orc.sw_contract(s, theta, x, ac)
    for k in list(range(7)) + [7 + q for q in PROBES]:
        hk = _step(theta, k, 1e-6)
        tp, tm = theta.copy(), theta.copy()
        tp[k] += hk
        tm[k] -= hk
        fd = ((orc.sw_forces(s, tp, x) - orc.sw_forces(s, tm, x)) * ac).sum() / (2 * hk)
        assert abs(th[k] - fd) <= _rtol(k) * max(abs(fd), 1e-4 * _gmax(th, k)), (k, th[k], fd)


def test_stress_loss_derivatives(crystal, theta):
    box, x, v = crystal
    s = orc.make_sw_system(len(x), box, mlp=True)
    L = orc.make_sw_loss(D.STRESS_WEIGHT)
    l, gx, gv, gp = orc.sw_loss_grad(s, theta, L, x, v)

    def loss(xx, pp):
        return orc.sw_loss_grad(s, pp, L, xx, v)[0]

    u = np.random.default_rng(6).normal(size=x.shape)
    h = 1e-6
    fd = (loss(x + h * u, theta) - loss(x - h * u, theta)) / (2 * h)
    assert abs((gx * u).sum() - fd) <= 1e-6 * abs(fd)
    for k in [0, 5] + [7 + q for q in PROBES]:
        hk = _step(theta, k, 1e-6)
        tp, tm = theta.copy(), theta.copy()
        tp[k] += hk
        tm[k] -= hk
        fd = (loss(x, tp) - loss(x, tm)) / (2 * hk)
        assert abs(gp[k] - fd) <= _rtol(k) * max(abs(fd), 1e-4 * _gmax(gp, k)), (k, gp[k], fd)


def test_reverse_gradient_equals_gradient_of_mean_loss(crystal, theta):
    """The reference's self-check run (diamond.jl:1910-1947: 12 steps, loss every 5,
    truncation 12) with the learned term: the start state is rebuilt and the reverse
    gradient of the MLP parameters equals central differences of the forward loss."""
    box, x, v = crystal
    s = orc.make_sw_system(len(x), box, mlp=True)
    seeds = np.arange(1, 13, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    L = orc.make_sw_loss(D.STRESS_WEIGHT)
    xf, vf, lf, sx, sv = orc.sw_forward_sim(s, theta, x, v, seeds, 4.0, 12, 5, 0.0005, L)
    xr, vr, lr, g = orc.sw_reverse_sim(s, theta, xf, vf, seeds, 4.0, 12, 5, 12, 0.0005, sx, sv, L)
    dx = xr - x
    dx -= np.round(dx / box) * box
    assert np.abs(dx).max() < 1e-8 and abs(lr - lf) <= 1e-10 * abs(lf)
    for k in [0, 6] + [7 + q for q in PROBES]:
        hk = _step(theta, k, 1e-5)
        tp, tm = theta.copy(), theta.copy()
        tp[k] += hk
        tm[k] -= hk
        lp = orc.sw_forward_sim(s, tp, x, v, seeds, 4.0, 12, 5, 0.0005, L)[2]
        lm = orc.sw_forward_sim(s, tm, x, v, seeds, 4.0, 12, 5, 0.0005, L)[2]
        fd = (lp - lm) / (2 * hk)
        assert abs(g[k] - fd) <= 1e-5 * max(abs(fd), 1e-3 * _gmax(g, k)), (k, g[k], fd)
