"""The oracle's Monte-Carlo barostat (MonteCarloBarostatNoUnits / apply_coupling!,
water.jl:789-865) against an independent numpy restatement of one attempt: the volume draw,
the molecule-centre scaling, the energy difference over the same pair list, the acceptance
rule and the step-size adaptation; plus rigid molecules under scaling and the direction of
a low-density box under 1 bar.
"""

import math

import numpy as np
import pytest

from oracle import orc
from revsim import constants as C, systems

BAR_NA = 0.0602214076   # kJ/mol per bar nm^3


def _scale_np(x, box, l):
    x = x.reshape(-1, 3, 3)
    d = x[:, 1:] - x[:, :1]
    d -= box * np.round(d / box)
    c = x[:, 0] + d.sum(axis=1) / 3.0
    xt = x + (c * l - c)[:, None, :]
    Ln = box * l
    return (xt - np.floor(xt / Ln) * Ln).reshape(-1, 3), Ln


def test_uniform_stream():
    u = np.array([orc.lib().orc_barostat_uniform(11, k) for k in range(20000)])
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 0.01 and abs(u.var() - 1 / 12) < 0.003
    assert orc.lib().orc_barostat_uniform(11, 5) == u[5]


@pytest.mark.parametrize("seed", [3, 4, 5, 6])
def test_attempt_matches_restatement(small_water, seed):
    n_mol, box, x, _ = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    pairs = orc.neighbor_pairs(s, x)
    b = orc.make_barostat(box, seed=seed)
    b.volume_scale = 0.4   # moves large enough to be rejected now and then
    u1 = orc.lib().orc_barostat_uniform(seed, 0)
    u2 = orc.lib().orc_barostat_uniform(seed, 1)
    E = orc.energy(s, p, x, pairs)
    V = box ** 3
    dV = 0.4 * (2 * u1 - 1)
    l = ((V + dV) / V) ** (1 / 3)
    xt, Ln = _scale_np(x, box, l)
    st = orc.make_system(n_mol, Ln)
    Et = orc.energy(st, p, xt, pairs)
    kT = C.KB * C.TEMP
    dW = (Et - E) + BAR_NA * dV - n_mol * kT * math.log((V + dV) / V)
    accept = dW <= 0 or u2 < math.exp(-dW / kT)
    acc, xo = orc.barostat_attempt(s, p, x, pairs, b)
    assert acc == accept and b.n_draws == 1 and b.n_attempted == 1
    if accept:
        assert abs(s.box - Ln) <= 1e-15 * Ln
        assert np.abs(xo - xt).max() <= 1e-12
    else:
        assert s.box == box and np.array_equal(xo, x)


def test_molecules_stay_rigid_under_scaling(small_water):
    n_mol, box, x, _ = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    pairs = orc.neighbor_pairs(s, x)
    b = orc.make_barostat(box, seed=1)
    for k in range(20):
        acc, x2 = orc.barostat_attempt(s, p, x, pairs, b)
        if acc:
            break
    assert acc and s.box != box

    def geom(xx, L):
        xx = xx.reshape(-1, 3, 3)
        d = xx[:, 1:] - xx[:, :1]
        d -= L * np.round(d / L)
        return np.linalg.norm(d, axis=2), np.einsum("ij,ij->i", d[:, 0], d[:, 1])
    r0, c0 = geom(x, box)
    r1, c1 = geom(x2, s.box)
    assert np.abs(r1 - r0).max() <= 1e-12 and np.abs(c1 - c0).max() <= 1e-12
    assert x2.min() >= 0 and x2.max() < s.box


@pytest.mark.parametrize("fixture,vs", [("small_water", 5.0), ("small_water", 0.05),
                                        ("dense_water", 5.0)])
def test_step_size_adaptation(request, fixture, vs):
    """After 10 attempts the volume step shrinks by scale_increment below 25 % accepted and
    grows (capped at max_volume_frac V) above 75 % (water.jl:851-861); the three cases hit
    the keep, grow and shrink branches."""
    n_mol, box, x, _ = request.getfixturevalue(fixture)
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    pairs = orc.neighbor_pairs(s, x)
    b = orc.make_barostat(box, seed=2)
    b.volume_scale = vs
    V0 = None
    for k in range(10):
        if k == 9:
            V0 = s.box ** 3
        _, x = orc.barostat_attempt(s, p, x, pairs, b)
    n = b.n_accepted_total
    if n < 2.5:
        assert abs(b.volume_scale - vs / 1.1) <= 1e-15 * vs and b.n_attempted == 0
    elif n > 7.5:
        assert abs(b.volume_scale - min(vs * 1.1, 0.3 * V0)) <= 1e-15 * vs and b.n_attempted == 0
    else:
        assert b.volume_scale == vs and b.n_attempted == 10


def test_low_density_box_shrinks_under_one_bar(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    b = orc.make_barostat(box, seed=7, n_steps=5)
    orc.forward_sim_barostat(s, p, x, v, systems.noise_seeds(200, seed=3), 1.0, 200, 0.001, b)
    assert b.n_draws == 40 and b.n_accepted_total > 5
    assert s.box < box
