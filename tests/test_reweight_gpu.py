"""The potential-energy parameter gradient (revsim_energy_grad) and the reweighting gradient
estimator (reweighting_sim, water.jl:1107-1210) against the FP64 oracle.

Bars: energy and dE/dtheta 1e-10 relative for every pair form (the kernel is FP64 in both
precision modes), 1e-9 with the learned term in FP64 mode; the estimator from the engine's
FP64 run equal to the oracle's estimator over the same seeded run to 1e-6 (relative to the
largest gradient entry), and its loss equal to the forward loss of the run (water.jl:1615).
"""

import numpy as np
import pytest

from oracle import orc
from revsim import Engine, constants as C, mlp, systems
from revsim.engine import RdfTerm
from revsim.water import forward_sim, reweighting_sim

pytestmark = pytest.mark.gpu

FORMS = ["lj", "dexp", "buck", "ljsc", "buff"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("form", FORMS)
def test_energy_gradient_matches_oracle(dense_water, form, prec):
    n_mol, box, x, v = dense_water
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    Eo, go = orc.energy_grads(s, p, x, orc.neighbor_pairs(s, x))
    e = Engine(n_mol, box, inter_type=form, precision=prec)
    e.set_params(p)
    e.set_state(x, v)
    E, g = e.energy_grad()
    e.close()
    assert abs(E[0] - Eo) <= 1e-10 * abs(Eo)
    assert np.abs(g[0] - go).max() <= 1e-10 * np.abs(go).max(), (g[0], go)


def test_energy_gradient_with_the_learned_term(dense_water):
    n_mol, box, x, v = dense_water
    th = mlp.init_params(3) + np.random.default_rng(4).normal(scale=0.05, size=mlp.N_PARAMS)
    p = np.concatenate([C.default_params("lj"), th])
    s = orc.make_system(n_mol, box, "lj", mlp=True)
    Eo, go = orc.energy_grads(s, p, x, orc.neighbor_pairs(s, x))
    e = Engine(n_mol, box, inter_type="lj", precision="fp64", mlp=True)
    e.set_params(p)
    e.set_state(x, v)
    E, g = e.energy_grad()
    e.close()
    assert abs(E[0] - Eo) <= 1e-9 * abs(Eo)
    assert np.abs(g[0, :7] - go[:7]).max() <= 1e-9 * np.abs(go[:7]).max()
    assert np.abs(g[0, 7:] - go[7:]).max() <= 1e-9 * np.abs(go[7:]).max()


def test_reweighting_estimator_matches_oracle(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box, "lj")
    p = np.array(C.default_params("lj"))
    n = 200
    t0 = orc.RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, 0.04, n, 0, 1, np.zeros(n), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    ot = orc.RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, 0.04, n, 0, 1, target, 2, 1.0)
    ol = orc.Loss([ot])
    n_steps, nl = 100, 20
    seeds = systems.noise_seeds(n_steps, seed=17)
    # oracle estimator over the same run (water.jl:1159-1201)
    xo, vo = x.copy(), v.copy()
    L, dE, LdE = 0.0, np.zeros(7), np.zeros(7)
    for b in range(n_steps // nl):
        xo, vo, lb, _, _ = orc.forward_sim(s, p, xo, vo, seeds[b * nl:(b + 1) * nl], 1.0, nl, nl,
                                          0.001, ol)
        _, gb = orc.energy_grads(s, p, xo, orc.neighbor_pairs(s, xo))
        L += lb
        dE += gb
        LdE += lb * gb
    nb = n_steps // nl
    beta = 1.0 / (C.KB * C.TEMP)
    g_ref = -beta * (LdE / nb - (L / nb) * dE / nb)
    term = RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, 0.04, n, 0, 1, target, 2, 1.0)
    sys, loss, grads, l_rdf, l_ev = reweighting_sim(x, v, box, seeds, 1.0, n_steps, nl, p, 0.001, 1,
                                                    "lj", "rdf", loss_terms=[term], precision="fp64")
    assert abs(loss - L / nb) <= 1e-8 * abs(L / nb)
    assert np.abs(grads - g_ref).max() <= 1e-6 * np.abs(g_ref).max(), (grads, g_ref)
    # the reference's check: the reweighting loss is the forward loss of the same run
    _, loss_fwd, _ = forward_sim(x, v, box, seeds, 1.0, n_steps, nl, p, 0.001, 1, "lj", "rdf",
                                 loss_terms=[term], precision="fp64")
    assert abs(loss - loss_fwd) <= 1e-9 * abs(loss_fwd)
    sys.engine.close()
