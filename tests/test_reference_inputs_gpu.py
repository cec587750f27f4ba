"""GPU parity on the reference's own inputs: the tip3p.pdb box (895 molecules, 3.0 nm,
water.jl:32) with every parameter set in water/trained_force_fields/*.xml, from the
committed fixture tests/golden/reference_inputs.npz, against the FP64 oracle.

Tolerances: neighbour pair set bit-exact; forces 1e-10 (FP64) / 1e-5 (mixed) relative,
norm-wise; force VJP 1e-10 / 1e-4; a 20-step forward + reverse gradient (gamma = 1/ps) 1e-6
(FP64) / 1e-4 (mixed LJ; 3e-4 for the exponential and soft-core forms, whose FP32
exponentials amplify the rounding of r) in units of dL/dlog(theta) floored at 1 % of the
largest component; the same run with the caller's noise (revsim_forward_noise) as well.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import Engine, RdfTerm, systems

from test_reference_inputs import SETS, load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def nrel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def scaled_err(g, ref, p):
    s = np.abs(ref * p)
    return np.abs((g - ref) * p) / np.maximum(s, 0.01 * s.max())


def test_tip3p_neighbor_pairs_bit_exact():
    x, box, sets = load()
    e = Engine(895, box)
    e.set_params(sets["tip3p"][1])
    e.set_state(x, np.zeros_like(x))
    np.testing.assert_array_equal(e.neighbor_pairs(0), orc.neighbor_pairs(orc.make_system(895, box), x))


@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_tip3p_forces_and_vjp(name, prec):
    x, box, sets = load()
    form, p = sets[name]
    rng = np.random.default_rng(17)
    w, ac = rng.normal(size=x.shape), rng.normal(size=x.shape)
    e = Engine(895, box, inter_type=form, precision=prec)
    e.set_params(p)
    e.set_state(x, np.zeros_like(x))
    F, G, th = e.force_vjp(w, ac)
    s = orc.make_system(895, box, form)
    Fo, Go, J = orc.forces_grads(s, p, x, orc.neighbor_pairs(s, x), w)
    assert nrel(e.forces(), Fo) < (1e-10 if prec == "fp64" else 1e-5)
    assert nrel(F, Fo) < (1e-10 if prec == "fp64" else 1e-5)
    assert nrel(G, Go) < (1e-10 if prec == "fp64" else 1e-4)
    tol = 1e-10 if prec == "fp64" else 1e-4
    assert np.all(scaled_err(th[0], ac.ravel() @ J, p) < tol)


@pytest.mark.parametrize("name", SETS)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("noise", ["seeds", "host"])
def test_tip3p_gradient_matches_oracle(name, prec, noise):
    x, box, sets = load()
    form, p = sets[name]
    s = orc.make_system(895, box, form)
    v = systems.mb_velocities(895, seed=3)
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    ol = orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
    n = 20
    seeds = systems.noise_seeds(n, seed=4)
    xi = None
    if noise == "host":
        rng = np.random.default_rng(6)
        m = np.where(np.arange(x.shape[0]) % 3 == 0, 15.99943, 1.007947)
        xi = rng.normal(size=(n,) + x.shape) * np.sqrt(0.00831446261815324 * s.temp / m)[None, :, None]
    xf, vf, lfo, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, ol, noise=xi)
    _, _, lro, go = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, ol, noise=xi)
    e = Engine(895, box, inter_type=form, precision=prec)
    e.set_params(p)
    e.set_loss([RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
    e.set_state(x, v)
    lf = e.forward(seeds, 1.0, n, n, 0.001, noise=xi)
    lr, g = e.reverse(seeds, 1.0, n, n, n, 0.001, noise=xi)
    assert abs(lf[0] - lfo) < (1e-10 if prec == "fp64" else 1e-5) * abs(lfo)
    tol = 1e-6 if prec == "fp64" else (1e-4 if form == "lj" else 3e-4)
    err = scaled_err(g[0], go, p)
    assert np.all(err < tol), err
