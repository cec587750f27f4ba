"""The FP64 CPU oracle of the Stillinger-Weber diamond path against independent checks.

The reference's diamond path needs Julia, Enzyme and JAX, none of which run here, and ships
no golden vectors, so the oracle is pinned by: an independent numpy restatement of the SW
energy (diamond.jl:348-381) on the same term set; F = -dU/dx; the Hessian-vector product,
dF/dtheta and every loss derivative vs central differences; the virial tensor vs the strain
derivative of the energy (the dU/dh box term of diamond.jl:681-704 plus -F^T R); and the
reference's own self-check (diamond.jl:1910-1942): 12 steps, loss every 5, truncation 12,
gamma 4/ps, dt 0.5 fs, where the reverse pass must rebuild the start state (< 1e-8) and its
gradient equals the gradient of the mean loss over the three loss points.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import diamond as D

P0 = D.default_params()


@pytest.fixture(scope="module")
def crystal():
    """216 atoms (3^3 cells) with 0.01 nm noise and 298 K velocities."""
    x, box = D.diamond_coords(3, noise=0.01, seed=4)
    v = D.mb_velocities(len(x), seed=5)
    s = orc.make_sw_system(len(x), box)
    return s, box, x, v


def _terms(x, box, p):
    """Independent term enumeration: (2-body pairs, 3-body (centre, j, k) triplets) with
    min-image displacements from the centre."""
    n = len(x)
    d = x[None, :, :] - x[:, None, :]
    d -= np.round(d / box) * box
    r = np.linalg.norm(d, axis=2)
    np.fill_diagonal(r, np.inf)
    nb = r < p[2] * p[5]
    pairs = [(i, j) for i in range(n) for j in range(i + 1, n) if nb[i, j]]
    trips = []
    for c in range(n):
        js = np.nonzero(nb[c])[0]
        for a in range(len(js)):
            for b in range(a + 1, len(js)):
                trips.append((c, js[a], js[b]))
    return d, pairs, trips


def _energy_np(d, pairs, trips, p, eps_strain=None):
    A, B, a, lam, gam, sig, eps = p
    M = np.eye(3) if eps_strain is None else np.eye(3) + eps_strain
    E = 0.0
    for i, j in pairs:
        s = np.linalg.norm(M @ d[i, j]) / sig
        E += eps * A * (B * s**-4 - 1.0) * np.exp(1.0 / (s - a))
    for c, j, k in trips:
        u, w = M @ d[c, j], M @ d[c, k]
        ru, rw = np.linalg.norm(u), np.linalg.norm(w)
        cs = u @ w / (ru * rw)
        E += eps * lam * np.exp(gam / (ru / sig - a) + gam / (rw / sig - a)) * (cs + 1 / 3) ** 2
    return E


def test_energy_matches_independent_restatement(crystal):
    s, box, x, _ = crystal
    d, pairs, trips = _terms(x, box, P0)
    assert len(pairs) > 0 and len(trips) > 0
    e_np = _energy_np(d, pairs, trips, P0)
    assert abs(orc.sw_energy(s, P0, x) - e_np) <= 1e-12 * abs(e_np)


def test_forces_are_minus_energy_gradient(crystal):
    s, box, x, _ = crystal
    F = orc.sw_forces(s, P0, x)
    u = np.random.default_rng(1).normal(size=x.shape)
    h = 1e-6
    dE = (orc.sw_energy(s, P0, x + h * u) - orc.sw_energy(s, P0, x - h * u)) / (2 * h)
    assert abs((F * u).sum() + dE) <= 1e-7 * abs(dE)
    assert np.abs(F.sum(axis=0)).max() <= 1e-9 * np.abs(F).max()   # momentum conservation


def test_force_vjp_matches_central_difference(crystal):
    s, box, x, _ = crystal
    rng = np.random.default_rng(2)
    w = rng.normal(size=x.shape)
    u = rng.normal(size=x.shape)
    _, G, _ = orc.sw_forces_grads(s, P0, x, w, jac=False)
    h = 1e-6
    fd = ((w / s.mass) * (orc.sw_forces(s, P0, x + h * u) - orc.sw_forces(s, P0, x - h * u))).sum() / (2 * h)
    assert abs((G * u).sum() - fd) <= 1e-6 * abs(fd)


@pytest.mark.parametrize("k", range(7))
def test_force_parameter_jacobian_matches_central_difference(crystal, k):
    s, box, x, _ = crystal
    _, _, J = orc.sw_forces_grads(s, P0, x, np.zeros_like(x))
    h = 1e-6 * abs(P0[k])
    pp, pm = P0.copy(), P0.copy()
    pp[k] += h
    pm[k] -= h
    fd = (orc.sw_forces(s, pp, x) - orc.sw_forces(s, pm, x)).ravel() / (2 * h)
    assert np.linalg.norm(J[:, k] - fd) <= 1e-6 * np.linalg.norm(fd)


def test_virial_is_strain_derivative_of_energy(crystal):
    s, box, x, v = crystal
    d, pairs, trips = _terms(x, box, P0)
    V = box**3
    W = orc.sw_stress(s, P0, x, v, vel_term=False) * V
    h = 1e-6
    for a in range(3):
        for b in range(3):
            e = np.zeros((3, 3))
            e[a, b] = h
            fd = (_energy_np(d, pairs, trips, P0, e) - _energy_np(d, pairs, trips, P0, -e)) / (2 * h)
            assert abs(W[a, b] - fd) <= 1e-7 * np.abs(W).max()
    # The kinetic tensor -sum m (v - vbar)(v - vbar)^T (diamond.jl:754-756).
    vb = v - v.mean(axis=0)
    K = -s.mass * vb.T @ vb
    assert np.allclose(orc.sw_stress(s, P0, x, v) * V, W + K, rtol=1e-13, atol=1e-9)
    # Isotropic scaling through the oracle's own energy: trace(W) = d E(lambda x, lambda L)/d lambda.
    lam = 1e-6
    sp = orc.make_sw_system(s.n_atoms, box * (1 + lam))
    sm = orc.make_sw_system(s.n_atoms, box * (1 - lam))
    fd = (orc.sw_energy(sp, P0, x * (1 + lam)) - orc.sw_energy(sm, P0, x * (1 - lam))) / (2 * lam)
    assert abs(np.trace(W) - fd) <= 1e-7 * abs(fd)


def test_stress_loss_gradients_match_central_differences(crystal):
    s, box, x, v = crystal
    rng = np.random.default_rng(3)
    L = orc.make_sw_loss(D.STRESS_WEIGHT, rng.normal(scale=50.0, size=9))
    val, gx, gv, gp = orc.sw_loss_grad(s, P0, L, x, v)
    loss = lambda xx, vv, pp: orc.sw_loss_grad(s, pp, L, xx, vv)[0]
    u = rng.normal(size=x.shape)
    h = 1e-6
    fd = (loss(x + h * u, v, P0) - loss(x - h * u, v, P0)) / (2 * h)
    assert abs((gx * u).sum() - fd) <= 1e-6 * abs(fd)
    fd = (loss(x, v + h * u, P0) - loss(x, v - h * u, P0)) / (2 * h)
    assert abs((gv * u).sum() - fd) <= 1e-6 * abs(fd)
    for k in range(7):
        hk = 1e-6 * abs(P0[k])
        pp, pm = P0.copy(), P0.copy()
        pp[k] += hk
        pm[k] -= hk
        fd = (loss(x, v, pp) - loss(x, v, pm)) / (2 * hk)
        assert abs(gp[k] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(gp).max())


def _selfcheck(crystal, n_steps=12, n_loss=5, n_trunc=12, gamma=4.0, dt=0.0005):
    s, box, x, v = crystal
    seeds = np.arange(1, n_steps + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    L = orc.make_sw_loss(D.STRESS_WEIGHT)
    xf, vf, lf, sx, sv = orc.sw_forward_sim(s, P0, x, v, seeds, gamma, n_steps, n_loss, dt, L)
    xr, vr, lr, g = orc.sw_reverse_sim(s, P0, xf, vf, seeds, gamma, n_steps, n_loss, n_trunc, dt,
                                       sx, sv, L)
    return s, x, v, seeds, L, lf, xr, vr, lr, g, len(sx)


def test_reference_selfcheck_reconstruction_and_loss(crystal):
    """diamond.jl:1939-1941: the start state is rebuilt and the reverse loss equals the
    forward loss (here to rounding, since both use the same exact term set)."""
    s, x, v, seeds, L, lf, xr, vr, lr, g, n_blocks = _selfcheck(crystal)
    assert n_blocks == 3
    box = s.box
    dx = xr - x
    dx -= np.round(dx / box) * box
    assert np.abs(dx).max() < 1e-8
    assert np.abs(vr - v).max() < 1e-8 * np.abs(v).max()
    assert abs(lr - lf) <= 1e-10 * abs(lf)


def test_reverse_gradient_equals_gradient_of_mean_loss(crystal):
    """With truncation >= n_steps every block's adjoint runs back to step 0, so the reverse
    gradient is d(mean loss)/dtheta of the forward pass (diamond.jl:1943-1947 compare it with
    the forward-mode AD gradient; central differences stand in for that here)."""
    s, x, v, seeds, L, lf, xr, vr, lr, g, _ = _selfcheck(crystal)
    for k in range(7):
        hk = 1e-5 * abs(P0[k])
        pp, pm = P0.copy(), P0.copy()
        pp[k] += hk
        pm[k] -= hk
        lp = orc.sw_forward_sim(s, pp, x, v, seeds, 4.0, 12, 5, 0.0005, L)[2]
        lm = orc.sw_forward_sim(s, pm, x, v, seeds, 4.0, 12, 5, 0.0005, L)[2]
        fd = (lp - lm) / (2 * hk)
        assert abs(g[k] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(g).max()), (k, g[k], fd)


def test_truncated_blocks_restart_from_snapshots(crystal):
    """Truncation 3 < n_steps_loss 5: each block runs back 3 steps from its loss point (2 for
    the loss point at step 2), then the state is restored from the forward snapshot
    (diamond.jl:1800-1860).  Each block's gradient is then the derivative of its loss through
    those steps with the state before them held fixed."""
    s, box, x, v = crystal
    seeds = np.arange(1, 13, dtype=np.uint64) * np.uint64(0x2545F4914F6CDD1D)
    L = orc.make_sw_loss(D.STRESS_WEIGHT)
    xf, vf, lf, sx, sv = orc.sw_forward_sim(s, P0, x, v, seeds, 4.0, 12, 5, 0.0005, L)
    xr, vr, lr, g = orc.sw_reverse_sim(s, P0, xf, vf, seeds, 4.0, 12, 5, 3, 0.0005, sx, sv, L)
    assert abs(lr - lf) <= 1e-10 * abs(lf)
    fd = np.zeros(7)
    for t in (12, 7, 2):
        n_back = t - max(t - 3 + 1, 1) + 1
        t0 = t - n_back
        x0, v0 = x, v
        if t0 > 0:
            x0, v0, _, _, _ = orc.sw_forward_sim(s, P0, x, v, seeds[:t0], 4.0, t0, t0, 0.0005)
        for k in range(7):
            hk = 1e-5 * abs(P0[k])
            pp, pm = P0.copy(), P0.copy()
            pp[k] += hk
            pm[k] -= hk
            lp = orc.sw_forward_sim(s, pp, x0, v0, seeds[t0:t], 4.0, n_back, n_back, 0.0005, L)[2]
            lm = orc.sw_forward_sim(s, pm, x0, v0, seeds[t0:t], 4.0, n_back, n_back, 0.0005, L)[2]
            fd[k] += (lp - lm) / (2 * hk) / 3
    for k in range(7):
        assert abs(g[k] - fd[k]) <= 1e-5 * max(abs(fd[k]), 1e-3 * np.abs(fd).max()), (k, g[k], fd[k])
