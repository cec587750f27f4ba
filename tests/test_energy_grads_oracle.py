"""The oracle's potential-energy parameter gradient (orc_energy_grads), the per-snapshot
dE/dtheta of the reference's reweighting estimator (water.jl:1176-1183), against central
differences of the oracle energy for every pair form, and for the learned pair correction."""

import numpy as np
import pytest

from oracle import orc
from revsim import constants as C, mlp

FORMS = ["lj", "dexp", "buck", "ljsc", "buff"]


@pytest.mark.parametrize("form", FORMS)
def test_energy_parameter_gradient_matches_central_difference(small_water, form):
    n_mol, box, x, _ = small_water
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    pairs = orc.neighbor_pairs(s, x)
    E, g = orc.energy_grads(s, p, x, pairs)
    assert abs(E - orc.energy(s, p, x, pairs)) <= 1e-12 * abs(E)
    for k in range(len(p)):
        h = 1e-6 * abs(p[k])
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (orc.energy(s, pp, x, pairs) - orc.energy(s, pm, x, pairs)) / (2 * h)
        # central differences of a ~1e4 kJ/mol energy resolve ~1e-8 |E| / |p_k|
        assert abs(g[k] - fd) <= 1e-6 * max(abs(fd), 1e-2 * abs(E) / abs(p[k])), (k, g[k], fd)


def test_energy_gradient_of_the_mlp_parameters(small_water):
    n_mol, box, x, _ = small_water
    s = orc.make_system(n_mol, box, "lj", mlp=True)
    th = mlp.init_params(3) + np.random.default_rng(4).normal(scale=0.05, size=mlp.N_PARAMS)
    p = np.concatenate([C.default_params("lj"), th])
    pairs = orc.neighbor_pairs(s, x)
    E, g = orc.energy_grads(s, p, x, pairs)
    assert g.shape == (7 + mlp.N_PARAMS,)
    for k in [0, 5, 7 + 3, 7 + 1088 + 70, 7 + 5248 + 3, 7 + 5312, 7 + mlp.PER_TYPE + 42,
              7 + 2 * mlp.PER_TYPE + 5300]:
        h = 1e-5 * max(abs(p[k]), 1.0)
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (orc.energy(s, pp, x, pairs) - orc.energy(s, pm, x, pairs)) / (2 * h)
        assert abs(g[k] - fd) <= 1e-6 * max(abs(fd), 1e-4 * abs(E)), (k, g[k], fd)
