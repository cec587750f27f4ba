"""The oracle's host-noise drivers (orc_forward_sim_hn / orc_reverse_sim_hn): fed the
per-step noise that the seeded drivers draw, they give the same trajectory, loss and
gradient bit for bit, and they use whatever noise they are given (water.jl:1033-1036,
1497-1498)."""

import numpy as np

from conftest import relaxed_water
from oracle import orc
from revsim import constants as C, systems


def _setup(n_mol=60, box=2.45, n=12):
    x, v = relaxed_water(n_mol, box, seed=2, steps=10)
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    loss = orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
    seeds = systems.noise_seeds(n, seed=5)
    return s, p, x, v, loss, seeds, n


def test_seed_noise_through_the_host_path_is_bit_identical():
    s, p, x, v, loss, seeds, n = _setup()
    xi = np.stack([orc.noise(s, int(sd)) for sd in seeds])
    a = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, loss)
    b = orc.forward_sim(s, p, x, v, None, 1.0, n, n, 0.001, loss, noise=xi)
    for u, w in zip(a, b):
        np.testing.assert_array_equal(u, w)
    ra = orc.reverse_sim(s, p, a[0], a[1], seeds, 1.0, n, n, n, 0.001, a[3], a[4], loss)
    rb = orc.reverse_sim(s, p, b[0], b[1], None, 1.0, n, n, n, 0.001, b[3], b[4], loss, noise=xi)
    for u, w in zip(ra, rb):
        np.testing.assert_array_equal(u, w)


def test_host_noise_is_used_and_reversed():
    s, p, x, v, loss, seeds, n = _setup()
    rng = np.random.default_rng(3)
    sd = np.sqrt(C.KB * s.temp / np.where(np.arange(x.shape[0]) % 3 == 0, C.O_MASS, C.H_MASS))
    xi = rng.normal(size=(n, x.shape[0], 3)) * sd[None, :, None]
    xs, vs, _, _, _ = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, loss)
    xf, vf, lf, sx, sv = orc.forward_sim(s, p, x, v, None, 1.0, n, n, 0.001, loss, noise=xi)
    assert np.abs(vf - vs).max() > 1e-3          # a different noise gives another trajectory
    x0, v0, lr, g = orc.reverse_sim(s, p, xf, vf, None, 1.0, n, n, n, 0.001, sx, sv, loss, noise=xi)
    d = x0 - x
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < 1e-9                # water.jl:1613
    assert abs(lr - lf) < 1e-7                   # water.jl:1614
    assert np.all(np.isfinite(g))
