"""The learned pair correction on the GPU (librevsim.so with ``mlp`` in the system
description) against the FP64 oracle (oracle/mlp_oracle.c inside revsim_oracle.c).

Bars: forces 1e-10 (FP64) / 1e-5 (mixed) relative; the VJP and the parameter contraction
sum_a acoef_a . dF_a/dtheta over all 15,946 parameters 1e-9 (FP64) / 1e-4 (mixed) relative to
the largest entry of each group (classical, each MLP layer); the reverse-pass gradient vs the
oracle's 1e-6 (a strongly-on MLP) / 1e-4 (an MLP of trained size; the classical group
parameter-scaled, as in the classical tests); with
zero MLP weights the forces equal the classical engine's; batched replicas give each replica
its own MLP gradient.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import Engine, constants as C, mlp, systems
from revsim.engine import RdfTerm

pytestmark = pytest.mark.gpu

PRECS = [("fp64", 1e-10, 1e-9), ("mixed", 1e-5, 1e-4)]


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


@pytest.fixture(scope="module")
def theta():
    """A strongly-on MLP: every weight and bias perturbed by N(0, 0.05)."""
    th = mlp.init_params(3)
    th += np.random.default_rng(4).normal(scale=0.05, size=th.shape)
    return np.concatenate([C.default_params("lj"), th])


@pytest.fixture(scope="module")
def theta_mild():
    """The seeded initialisation perturbed by N(0, 0.005): pair energies of the size a trained
    correction has.  The strongly-on MLP above makes short-range O-H and H-H forces so stiff
    that FP32 rounding grows to ~1e-3 in the bonded-parameter gradients over 30 steps."""
    th = mlp.init_params(3)
    th += np.random.default_rng(4).normal(scale=0.005, size=th.shape)
    return np.concatenate([C.default_params("lj"), th])


def nrel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def groups(n):
    """Index groups of the parameter vector: classical, then per type W1+b1, W2+b2, w3+b3."""
    out = [np.arange(7)]
    for t in range(3):
        o = 7 + t * mlp.PER_TYPE
        a = mlp.H * mlp.NRBF + mlp.H
        b = a + mlp.H * mlp.H + mlp.H
        out += [np.arange(o, o + a), np.arange(o + a, o + b), np.arange(o + b, o + mlp.PER_TYPE)]
    return out


def group_errs(g, ref, theta=None):
    """Per group: max |g - ref| / max |ref|; for the classical group, when theta is given,
    the parameter-scaled error of the classical tests (the seven parameters span eight
    decades): max |(g - ref) theta| / max(|ref theta|, 0.01 max |ref theta|)."""
    out = []
    for k, ix in enumerate(groups(len(ref))):
        if k == 0 and theta is not None:
            sc = np.abs(ref[ix] * theta[ix])
            out.append(float((np.abs((g[ix] - ref[ix]) * theta[ix]) / np.maximum(sc, 0.01 * sc.max())).max()))
        else:
            out.append(float(np.abs(g[ix] - ref[ix]).max() / np.abs(ref[ix]).max()))
    return out


def group_err(g, ref):
    return max(group_errs(g, ref))


def _engine(n_mol, box, prec, theta, **kw):
    e = Engine(n_mol, box, inter_type="lj", precision=prec, mlp=True, **kw)
    assert e.n_params == 7 + mlp.N_PARAMS
    e.set_params(theta)
    return e


@pytest.mark.parametrize("prec,ftol,gtol", PRECS)
def test_forces_vjp_and_contraction(dense_water, theta, prec, ftol, gtol):
    n_mol, box, x, v = dense_water
    rng = np.random.default_rng(7)
    w = rng.normal(size=x.shape)
    ac = rng.normal(size=x.shape)
    s = orc.make_system(n_mol, box, "lj", mlp=True)
    pairs = orc.neighbor_pairs(s, x)
    Fo, Go, _ = orc.forces_grads(s, theta, x, pairs, w, jac=False)
    tho = orc.contract(s, theta, x, pairs, ac)
    e = _engine(n_mol, box, prec, theta)
    e.set_state(x, v)
    F, G, th = e.force_vjp(w, ac)
    F2 = e.forces()
    e.close()
    F0 = orc.forces(orc.make_system(n_mol, box, "lj"), theta[:7], x, pairs)
    assert nrel(Fo, F0) > 1e-3                     # the learned term is on
    assert nrel(F, Fo) <= ftol
    assert np.array_equal(F, F2)
    assert nrel(G, Go) <= gtol
    assert group_err(th[0], tho) <= gtol, group_err(th[0], tho)


def test_learned_term_off_is_the_classical_engine(dense_water):
    n_mol, box, x, v = dense_water
    p = np.concatenate([C.default_params("lj"), np.zeros(mlp.N_PARAMS)])
    e = _engine(n_mol, box, "mixed", p)
    e.set_state(x, v)
    F1 = e.forces()
    e.close()
    e0 = Engine(n_mol, box, inter_type="lj", precision="mixed")
    e0.set_params(C.default_params("lj"))
    e0.set_state(x, v)
    F0 = e0.forces()
    e0.close()
    assert nrel(F1, F0) < 1e-6   # zero weights: u = 0 exactly, the forces differ by rounding order only


@pytest.mark.parametrize("prec,ftol,gtol", [("fp64", 1e-10, 1e-6), ("mixed", 1e-5, 1e-4)])
def test_reverse_gradient_matches_oracle(small_water, theta, theta_mild, prec, ftol, gtol):
    n_mol, box, x, v = small_water
    theta = theta if prec == "fp64" else theta_mild
    s = orc.make_system(n_mol, box, "lj", mlp=True)
    n = 200
    t0 = orc.RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, 0.04, n, 0, 1, np.zeros(n), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    ol = orc.Loss([orc.RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, 0.04, n, 0, 1, target, 2, 1.0)])
    steps = 30
    seeds = systems.noise_seeds(steps, seed=41)
    xf, vf, lfo, sx, sv = orc.forward_sim(s, theta, x, v, seeds, 1.0, steps, steps, 0.001, ol)
    _, _, lro, go = orc.reverse_sim(s, theta, xf, vf, seeds, 1.0, steps, steps, steps, 0.001, sx, sv, ol)
    e = _engine(n_mol, box, prec, theta)
    e.set_loss([RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, 0.04, n, 0, 1, target, 2, 1.0)])
    e.set_state(x, v)
    lf = e.forward(seeds, 1.0, steps, steps, 0.001)
    lr, g = e.reverse(seeds, 1.0, steps, steps, steps, 0.001)
    e.close()
    assert abs(lf[0] - lfo) <= ftol * abs(lfo) * (1 if prec == "fp64" else 10)
    assert abs(lr[0] - lf[0]) <= 1e-7 * abs(lf[0])
    errs = group_errs(g[0], go, theta)
    assert max(errs) <= gtol, errs


def test_batched_replicas_have_their_own_mlp_gradients(small_water, theta):
    n_mol, box, x, v = small_water
    seeds = systems.noise_seeds(20, seed=5)
    n = 200
    target = np.linspace(0.2, 1.2, n)
    term = RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, 0.04, n, 0, 1, target, 2, 1.0)
    e1 = _engine(n_mol, box, "fp64", theta)
    e1.set_loss([term])
    e1.set_state(x, v)
    e1.forward(seeds, 1.0, 20, 20, 0.001)
    _, g1 = e1.reverse(seeds, 1.0, 20, 20, 20, 0.001)
    e1.close()
    e2 = _engine([n_mol, n_mol], [box, box], "fp64", theta)
    e2.set_loss([term])
    x2 = np.concatenate([x, x])
    e2.set_state(x2, np.concatenate([v, v]))
    e2.forward(np.repeat(seeds[:, None], 2, axis=1), 1.0, 20, 20, 0.001)
    _, g2 = e2.reverse(np.repeat(seeds[:, None], 2, axis=1), 1.0, 20, 20, 20, 0.001)
    e2.close()
    for r in range(2):
        assert group_err(g2[r], g1[0]) <= 1e-9
