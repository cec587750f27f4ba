"""The exactly reversible integrator (revsim_set_integrator REVSIM_INTEGRATOR_EXACT).

* gamma = 0: 1,000 forward + 1,000 reverse steps (one untruncated block, the benchmark's)
  rebuild the start state bit for bit in FP64 and in mixed precision, where the reference's
  arithmetic rebuilds it only to rounding that the dynamics amplify (FP64 ~1e-8 nm, mixed up
  to ~0.1 nm);
* it stays the reference's dynamics: over 30 steps the trajectory within 1e-9 nm and the
  reverse-pass gradient within 1e-6 (FP64, dL/dlog(theta) units floored at 1 %) of the FP64
  oracle, the state and box differing from the reference's by the grid rounding (<= 2^-49 nm);
* gamma = 1/ps: the reverse pass rebuilds 100 steps to < 1e-9 nm (FP64), the O step's inverse
  being approximate as in the reference.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import Engine, RdfTerm, constants as C, systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def _grid(y):
    return np.rint(y * 2.0 ** 48) * 2.0 ** -48


def _terms(x, n_mol, box):
    s = orc.make_system(n_mol, box)
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    return target, [RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_exact_reversal_over_1000_steps(dense_water, prec):
    n_mol, box, x, v = dense_water
    _, terms = _terms(x, n_mol, box)
    e = Engine(n_mol, box, precision=prec)
    e.set_params(C.default_params())
    e.set_loss(terms)
    e.set_integrator("exact")
    e.set_state(x, v)
    e.autotune()
    e.set_state(x, v)
    n = 1000
    seeds = systems.noise_seeds(n, seed=3)
    lf = e.forward(seeds, 0.0, n, n, 0.001)
    # the forward pass started from the state on the grid (positions wrapped into the grid box)
    L = _grid(box)
    xq, vq = _grid(x), _grid(v)
    xq = xq - np.floor(xq / L) * L
    xq = np.where(xq < 0, xq + L, np.where(xq >= L, xq - L, xq))
    lr, g = e.reverse(seeds, 0.0, n, n, n, 0.001)
    x0, v0 = e.get_state()
    np.testing.assert_array_equal(x0, xq)
    np.testing.assert_array_equal(v0, vq)
    assert abs(lr[0] - lf[0]) <= 1e-12 * abs(lf[0])
    assert np.all(np.isfinite(g))


def test_exact_integrator_follows_the_oracle(small_water):
    n_mol, box, x, v = small_water
    target, terms = _terms(x, n_mol, box)
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    ol = orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
    n = 30
    seeds = systems.noise_seeds(n, seed=4)
    xf, vf, lfo, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, ol)
    _, _, _, go = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, ol)
    e = Engine(n_mol, box)
    e.set_params(p)
    e.set_loss(terms)
    e.set_integrator("exact")
    e.set_state(x, v)
    lf = e.forward(seeds, 1.0, n, n, 0.001)
    xg, _ = e.get_state()
    d = xg - xf
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-9
    assert abs(lf[0] - lfo) < 1e-9 * abs(lfo)
    _, g = e.reverse(seeds, 1.0, n, n, n, 0.001)
    sc = np.abs(go * p)
    assert np.all(np.abs((g[0] - go) * p) / np.maximum(sc, 0.01 * sc.max()) < 1e-6)


def test_exact_integrator_with_friction(small_water):
    n_mol, box, x, v = small_water
    _, terms = _terms(x, n_mol, box)
    e = Engine(n_mol, box)
    e.set_params(C.default_params())
    e.set_loss(terms)
    e.set_integrator("exact")
    e.set_state(x, v)
    n = 100
    seeds = systems.noise_seeds(n, seed=5)
    e.forward(seeds, 1.0, n, n, 0.001)
    e.reverse(seeds, 1.0, n, n, n, 0.001)
    x0, _ = e.get_state()
    d = x0 - x
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-9
    e.set_integrator("reference")
    with pytest.raises(Exception):
        e.reverse(seeds, 1.0, n, n, n, 0.001)   # the mode change invalidated the record
