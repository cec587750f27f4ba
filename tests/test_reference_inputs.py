"""The reference's own inputs: water/tip3p.pdb (the 895-molecule, 3.0 nm box of
water.jl:32) and the parameter sets it trained, water/trained_force_fields/*.xml, as stored
in tests/golden/reference_inputs.npz by tests/golden/make_reference_inputs.py.

CPU: the fixture matches the reference files when they are present; the oracle, started
from the PDB positions with each trained parameter set, satisfies the reference's own
self-check (water.jl:1613-1614: the start state rebuilt to < 1e-9 nm, |L_rev - L_fwd| <
1e-7) and its forces are minus the gradient of its energy.
"""

import os

import numpy as np
import pytest

from oracle import orc
from revsim import systems

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "reference_inputs.npz")
REF_WATER = "/root/reference/water"
SETS = ["tip3p", "lj", "lj_reweighting", "buckingham", "double_exponential", "lj_soft_core"]


def load():
    d = np.load(FIXTURE)
    return d["x_tip3p"], float(d["box_tip3p"]), {k: (str(d[f"form_{k}"]), d[f"params_{k}"]) for k in SETS}


@pytest.mark.skipif(not os.path.isdir(REF_WATER), reason="the reference tree is not on this machine")
def test_fixture_matches_the_reference_files():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mri", os.path.join(HERE, "golden", "make_reference_inputs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    fresh = mod.make(REF_WATER)
    d = np.load(FIXTURE)
    assert sorted(fresh) == sorted(d.files)
    for k in d.files:
        np.testing.assert_array_equal(fresh[k], d[k])


def test_fixture_shape():
    x, box, sets = load()
    assert x.shape == (2685, 3) and box == 3.0
    assert np.all((x >= 0) & (x < box))
    d = x[1::3] - x[0::3]
    d -= box * np.round(d / box)
    r = np.linalg.norm(d, axis=1)
    assert np.all(np.abs(r - 0.09572) < 5e-4)      # TIP3P O-H bonds
    assert sets["tip3p"][1][:2].tolist() == [0.31507524065751241, 0.635968]


@pytest.mark.parametrize("name", SETS)
def test_oracle_self_check_on_tip3p(name):
    x, box, sets = load()
    form, p = sets[name]
    s = orc.make_system(895, box, form)
    v = systems.mb_velocities(895, seed=3)
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    loss = orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
    n = 8
    seeds = systems.noise_seeds(n, seed=4)
    xf, vf, lf, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, loss)
    x0, v0, lr, g = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, loss)
    d = x0 - x
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-9
    assert abs(lr - lf) < 1e-7
    assert np.all(np.isfinite(g))


@pytest.mark.parametrize("name", ["lj", "buckingham", "double_exponential", "lj_soft_core"])
def test_oracle_forces_are_minus_energy_gradient_on_tip3p(name):
    x, box, sets = load()
    form, p = sets[name]
    s = orc.make_system(895, box, form)
    pairs = orc.neighbor_pairs(s, x)
    F = orc.forces(s, p, x, pairs)
    rng = np.random.default_rng(5)
    for a in rng.choice(x.shape[0], 4, replace=False):
        for u in range(3):
            def cd(h):
                xp, xm = x.copy(), x.copy()
                xp[a, u] += h
                xm[a, u] -= h
                return -(orc.energy(s, p, xp, pairs) - orc.energy(s, p, xm, pairs)) / (2 * h)
            # Richardson-extrapolated central difference (the stiff O-H bonds make the plain
            # one's h^2 error visible); rounding of the ~3e4 kJ/mol total limits it to ~1e-5
            fd = (4 * cd(2e-6) - cd(4e-6)) / 3
            assert abs(fd - F[a, u]) < 1e-4 + 1e-6 * abs(F[a, u]), (a, u, fd, F[a, u])
