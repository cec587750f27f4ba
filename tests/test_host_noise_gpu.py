"""The host-noise entry points (revsim_forward_noise / revsim_reverse_noise) on the GPU.

The reference draws each step's Langevin noise on the host (generate_noise!,
water.jl:867-873) and uses it at water.jl:1033-1036 (forward) and 1497-1498 (reverse).
A caller that passes that noise gets the reference's own trajectory:
* noise equal to the engine's own Philox draws gives the seeded entry points' trajectory bit
  for bit (FP64 and mixed), and their losses and gradients to 1e-12 (the smoothed-RDF
  histogram sums with FP64 atomics, whose order varies in the last bits);
* arbitrary caller noise: trajectory within 1e-10 nm, loss within 1e-10 relative and the
  gradient within 1e-6 (FP64) / 1e-4 (mixed) of the FP64 oracle fed the same noise, in
  units of dL/dlog(theta) floored at 1 % of the largest component;
* replicas: the noise of a step concatenates the replicas' atoms.
"""

import numpy as np
import pytest

from conftest import relaxed_water
from oracle import orc
from revsim import Engine, RdfTerm, RevsimError, constants as C, systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def _loss(x, s):
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    return (orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)]),
            [RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])


def _noise(n_steps, n_mol, temp, seed):
    rng = np.random.default_rng(seed)
    m = np.where(np.arange(3 * n_mol) % 3 == 0, C.O_MASS, C.H_MASS)
    return rng.normal(size=(n_steps, 3 * n_mol, 3)) * np.sqrt(C.KB * temp / m)[None, :, None]


def _scaled_err(g, ref, p):
    s = np.abs(ref * p)
    return np.abs((g - ref) * p) / np.maximum(s, 0.01 * s.max())


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_engine_noise_through_the_host_path_is_bit_identical(small_water, prec):
    n_mol, box, x, v = small_water
    _, terms = _loss(x, orc.make_system(n_mol, box))
    n = 40
    seeds = systems.noise_seeds(n, seed=9)
    out = []
    for host in (False, True):
        e = Engine(n_mol, box, precision=prec)
        e.set_params(C.default_params())
        e.set_loss(terms)
        xi = np.stack([e.noise([sd]) for sd in seeds]) if host else None
        e.set_state(x, v)
        lf = e.forward(None if host else seeds, 1.0, n, 20, 0.001, noise=xi)
        xf, vf = e.get_state()
        lr, g = e.reverse(None if host else seeds, 1.0, n, 20, 10, 0.001, noise=xi)
        x0, v0 = e.get_state()
        out.append((lf, xf, vf, lr, g, x0, v0))
        e.close()
    (lf, xf, vf, lr, g, x0, v0), (lf2, xf2, vf2, lr2, g2, x02, v02) = out
    for a, b in ((xf, xf2), (vf, vf2), (x0, x02), (v0, v02)):
        np.testing.assert_array_equal(a, b)
    for a, b in ((lf, lf2), (lr, lr2), (g, g2)):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-6), ("mixed", 1e-4)])
def test_host_noise_matches_oracle(small_water, prec, tol):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    ol, terms = _loss(x, s)
    n = 30
    xi = _noise(n, n_mol, s.temp, seed=11)
    xfo, vfo, lfo, sx, sv = orc.forward_sim(s, p, x, v, None, 1.0, n, n, 0.001, ol, noise=xi)
    x0o, _, lro, go = orc.reverse_sim(s, p, xfo, vfo, None, 1.0, n, n, n, 0.001, sx, sv, ol, noise=xi)
    e = Engine(n_mol, box, precision=prec)
    e.set_params(p)
    e.set_loss(terms)
    e.set_state(x, v)
    lf = e.forward(None, 1.0, n, n, 0.001, noise=xi)
    xf, _ = e.get_state()
    lr, g = e.reverse(None, 1.0, n, n, n, 0.001, noise=xi)
    x0, _ = e.get_state()
    d = xf - xfo
    d -= box * np.round(d / box)
    if prec == "fp64":
        assert np.abs(d).max() < 1e-10
        assert abs(lf[0] - lfo) < 1e-10 * abs(lfo)
    else:
        assert np.abs(d).max() < 1e-5
        assert abs(lf[0] - lfo) < 1e-5 * abs(lfo)
    r = x0 - x
    r -= box * np.round(r / box)
    assert np.abs(r).max() < (1e-9 if prec == "fp64" else 1e-7)
    assert np.all(_scaled_err(g[0], go, p) < tol), _scaled_err(g[0], go, p)


def test_host_noise_replicas_match_single_runs():
    sizes, boxes, temps = [150, 90], [2.6, 2.5], [285.0, 310.0]
    xs, vs = zip(*[relaxed_water(m, b, seed=90 + i, steps=20) for i, (m, b) in enumerate(zip(sizes, boxes))])
    n = 20
    xis = [_noise(n, m, t, seed=100 + i) for i, (m, t) in enumerate(zip(sizes, temps))]
    targets = [_loss(xs[r], orc.make_system(sizes[r], boxes[r]))[1][0].target for r in range(2)]
    eb = Engine(sizes, boxes, temp=temps)
    eb.set_params(C.default_params())
    eb.set_loss([RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.stack(targets), 2, 1.0)])
    eb.set_state(np.concatenate(xs), np.concatenate(vs))
    xi_b = np.concatenate(xis, axis=1)
    eb.forward(None, 1.0, n, n, 0.001, noise=xi_b)
    _, gb = eb.reverse(None, 1.0, n, n, n, 0.001, noise=xi_b)
    for r in range(2):
        e = Engine(sizes[r], boxes[r], temp=temps[r])
        e.set_params(C.default_params())
        e.set_loss([RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, targets[r], 2, 1.0)])
        e.set_state(xs[r], vs[r])
        e.forward(None, 1.0, n, n, 0.001, noise=xis[r])
        _, g = e.reverse(None, 1.0, n, n, n, 0.001, noise=xis[r])
        assert np.all(_scaled_err(gb[r], g[0], np.array(C.default_params())) < 1e-10)


def test_host_noise_argument_checks(small_water):
    n_mol, box, x, v = small_water
    e = Engine(n_mol, box)
    e.set_params(C.default_params())
    e.set_state(x, v)
    with pytest.raises(ValueError):
        e.forward(None, 1.0, 10, 10, 0.001, calc_loss=False, noise=np.zeros((9, 3 * n_mol, 3)))
    import ctypes
    rc = e._L.revsim_forward_noise(e.handle, None, 1.0, 10, 10, 0.001, 0, None)
    assert rc == -1
    # the handle stays usable
    e.forward(None, 1.0, 10, 10, 0.001, calc_loss=False, noise=np.zeros((10, 3 * n_mol, 3)))
    with pytest.raises(RevsimError):
        e._check(e._L.revsim_reverse_noise(e.handle, None, 1.0, 10, 10, 10, 0.001, np.inf, None, None))
