"""The FP64 CPU oracle against the reference's own identities and central differences.

The reference ships no golden vectors and cannot run here (Julia), so the oracle is
pinned by: F = -dU/dx; every derivative vs central FD / Richardson extrapolation (the
diffusion.jl:1659-1667 pattern); trajectory reconstruction < 1e-9 and
|L_rev - L_fwd| < 1e-7 (water.jl:1613-1614); the reverse gradient vs FD of the
forward loss for one loss block, and vs the mean of per-block FD gradients for
several blocks (the reference resets the adjoints at each block, water.jl:1541-1545).
"""

import numpy as np
import pytest

from oracle import orc
from revsim import constants as C, systems

FORMS = ["lj", "dexp", "buck", "ljsc", "buff"]


def _perturbed(small_water, scale=0.004, seed=5):
    n_mol, box, x, v = small_water
    rng = np.random.default_rng(seed)
    x = x + rng.normal(scale=scale, size=x.shape)
    return n_mol, box, x - np.floor(x / box) * box, v


@pytest.mark.parametrize("form", FORMS)
def test_forces_are_minus_energy_gradient(small_water, form):
    n_mol, box, x, _ = _perturbed(small_water)
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    pairs = orc.neighbor_pairs(s, x)
    F = orc.forces(s, p, x, pairs)
    u = np.random.default_rng(1).normal(size=x.shape)
    h = 1e-7
    dE = (orc.energy(s, p, x + h * u, pairs) - orc.energy(s, p, x - h * u, pairs)) / (2 * h)
    assert abs((F * u).sum() + dE) <= 1e-8 * abs(dE)


@pytest.mark.parametrize("form", FORMS)
def test_param_jacobian_and_vjp_match_fd(small_water, form):
    n_mol, box, x, _ = _perturbed(small_water)
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    pairs = orc.neighbor_pairs(s, x)
    rng = np.random.default_rng(2)
    w = rng.normal(size=x.shape)
    F, G, J = orc.forces_grads(s, p, x, pairs, w)
    F0 = orc.forces(s, p, x, pairs)
    assert np.abs(F - F0).max() <= 1e-13 * np.abs(F0).max()
    for k in range(len(p)):
        def fd(hr):
            dp = np.zeros_like(p)
            dp[k] = hr * abs(p[k])
            return (orc.forces(s, p + dp, x, pairs) - orc.forces(s, p - dp, x, pairs)).ravel() / (2 * dp[k])
        rich = (4 * fd(5e-5) - fd(1e-4)) / 3
        err = np.abs(rich - J[:, k]).max() / np.abs(J[:, k]).max()
        assert err < 5e-5, (form, k, err)
    # VJP: G . u = d/de sum_a (w_a/m_a) . F_a(x + e u)
    m = systems.masses(n_mol)[:, None]
    u = rng.normal(size=x.shape)
    hh = 1e-7
    phi = lambda xx: ((w / m) * orc.forces(s, p, xx, pairs)).sum()
    fd = (phi(x + hh * u) - phi(x - hh * u)) / (2 * hh)
    assert abs((G * u).sum() - fd) <= 1e-6 * abs(fd)


def test_neighbor_pairs_definition(small_water):
    n_mol, box, x, _ = small_water
    s = orc.make_system(n_mol, box)
    pairs = orc.neighbor_pairs(s, x)
    assert np.all(pairs[:, 0] < pairs[:, 1])
    assert np.all(pairs[:, 0] // 3 != pairs[:, 1] // 3)
    # brute force with numpy minimum image (same per-component folding)
    i, j = np.triu_indices(3 * n_mol, 1)
    keep = i // 3 != j // 3
    i, j = i[keep], j[keep]
    d = x[j] - x[i]
    d = np.where(d > box / 2, d - box, np.where(d < -box / 2, d + box, d))
    r2 = (d * d).sum(1)
    ref = set(zip(i[r2 <= 1.44].tolist(), j[r2 <= 1.44].tolist()))
    got = set(map(tuple, pairs.tolist()))
    sym = ref ^ got
    # only pairs within rounding of the cutoff may differ between the two foldings
    for a, b in sym:
        dd = x[b] - x[a]
        dd = np.where(dd > box / 2, dd - box, np.where(dd < -box / 2, dd + box, dd))
        assert abs((dd * dd).sum() - 1.44) < 1e-12


def test_noise_statistics():
    s = orc.make_system(2000, 6.0, temp=300.0)
    xi = np.concatenate([orc.noise(s, seed) for seed in (1, 2, 3)])
    m = np.tile(systems.masses(2000), 3)[:, None]
    z = xi / np.sqrt(C.KB * 300.0 / m)
    assert abs(z.mean()) < 0.02 and abs(z.var() - 1) < 0.02
    np.testing.assert_array_equal(orc.noise(s, 7), orc.noise(s, 7))
    assert not np.array_equal(orc.noise(s, 7), orc.noise(s, 8))


def _smooth_loss(s, x, width_cut=0.14):
    term0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, width_cut, 200, 0, 1, np.zeros(200), 2, 1.0)
    h = orc.rdf(s, term0, x)
    return orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, width_cut, 200, 0, 1, 0.9 * h + 0.05, 2, 1.0)])


def test_rdf_loss_gradient_fd(small_water):
    n_mol, box, x, _ = small_water
    s = orc.make_system(n_mol, box)
    for cut in (0.04, 0.14):
        loss = _smooth_loss(s, x, cut)
        _, g = orc.loss_grad(s, loss, x)
        u = np.random.default_rng(3).normal(size=x.shape)
        h = 1e-7
        fd = (orc.loss_grad(s, loss, x + h * u, False)[0] - orc.loss_grad(s, loss, x - h * u, False)[0]) / (2 * h)
        assert abs((g * u).sum() - fd) <= 1e-5 * abs(fd)


def test_rdf_normalisation_ideal_gas():
    # uniform random points: g(r) ~ 1 away from r = 0
    rng = np.random.default_rng(0)
    n_mol, box = 3000, 5.0
    x = rng.uniform(0, box, size=(3 * n_mol, 3))
    s = orc.make_system(n_mol, box)
    t = orc.RdfTerm(0, 0, 0.02, 0.02, 0.0005, 0.04, 100, 0, 1, np.zeros(100), 2, 1.0)
    h = orc.rdf(s, t, x)
    assert abs(h[20:].mean() - 1) < 0.05


@pytest.mark.parametrize("gamma", [1.0, 0.0])
def test_reconstruction_and_loss_identity(small_water, gamma):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    loss = _smooth_loss(s, x, 0.04)
    seeds = systems.noise_seeds(40, seed=11)
    xf, vf, lf, sx, sv = orc.forward_sim(s, p, x, v, seeds, gamma, 40, 40, 0.001, loss)
    xr, vr, lr, g = orc.reverse_sim(s, p, xf, vf, seeds, gamma, 40, 40, 40, 0.001, sx, sv, loss)
    d = xr - x
    d = np.where(d > box / 2, d - box, np.where(d < -box / 2, d + box, d))
    assert np.abs(d).max() < 1e-9          # water.jl:1613
    assert abs(lr - lf) < 1e-7             # water.jl:1614
    assert np.all(np.isfinite(g))


def _fd_loss_grad(s, p, x, v, seeds, gamma, n, loss, rels=(1e-6, 5e-7, 2e-7, 1e-7, 5e-8)):
    """Central differences of the forward loss, median over several step sizes: the
    loss has jumps where a pair crosses the 1.0 nm force cutoff (the reaction-field
    force is not zero there), which can poison any single step size."""
    out = []
    for k in range(len(p)):
        ds = []
        for rel in rels:
            dp = np.zeros_like(p)
            dp[k] = rel * abs(p[k])
            lp = orc.forward_sim(s, p + dp, x, v, seeds, gamma, n, n, 0.001, loss)[2]
            lm = orc.forward_sim(s, p - dp, x, v, seeds, gamma, n, n, 0.001, loss)[2]
            ds.append((lp - lm) / (2 * dp[k]))
        out.append(np.median(ds))
    return np.array(out)


def _scaled_err(g, fd, p):
    """|g - fd| in units of dL/dlog(theta), floored at 1% of the largest component."""
    sg, sf = np.abs(g * p), np.abs(fd * p)
    floor = 0.01 * sf.max()
    return np.abs((g - fd) * p) / np.maximum(sf, floor)


@pytest.mark.parametrize("form", ["lj", "dexp", "buck"])
def test_reverse_gradient_matches_fd_single_block(small_water, form):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    loss = _smooth_loss(s, x, 0.14)
    n = 20
    seeds = systems.noise_seeds(n, seed=4)
    xf, vf, lf, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, loss)
    _, _, _, g = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, loss)
    fd = _fd_loss_grad(s, p, x, v, seeds, 1.0, n, loss)
    err = _scaled_err(g, fd, p)
    assert np.all(err < 3e-4), err


def test_reverse_gradient_multi_block_is_mean_of_block_gradients(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    loss = _smooth_loss(s, x, 0.14)
    n, nl = 30, 10
    seeds = systems.noise_seeds(n, seed=5)
    xf, vf, lf, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, nl, 0.001, loss, n_steps_log=10)
    _, _, lr, g = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, nl, 0.001, sx, sv, loss, n_steps_log=10)
    assert abs(lr - lf) < 1e-7
    fds = [_fd_loss_grad(s, p, sx[b].reshape(-1, 3), sv[b].reshape(-1, 3), seeds[b * nl:(b + 1) * nl],
                         1.0, nl, loss) for b in range(3)]
    fd = sum(fds) / 3
    err = _scaled_err(g, fd, p)
    assert np.all(err < 3e-4), err


def test_reverse_rejects_trunc_longer_than_block(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    loss = _smooth_loss(s, x)
    _, _, lr, _ = orc.reverse_sim(s, p, x, v, systems.noise_seeds(10), 1.0, 10, 5, 6, 0.001,
                                  x.reshape(1, -1), v.reshape(1, -1), loss)
    assert np.isnan(lr)
