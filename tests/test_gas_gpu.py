"""Parity of the gas-in-water engine (include/revsim_gas.h) with the FP64 oracle of
diffusion.jl: forces, the force VJP and dF/dtheta contraction, the energy and dE/dtheta for
every pair form; the forward trajectory, gas centres and loss; the reverse pass's
reconstruction, loss and gradient, with and without truncation; and the argument checks."""

import numpy as np
import pytest

from conftest import relaxed_gas
from oracle import orc
from revsim import RevsimError, systems
from revsim.gas import GasEngine, forward_sim, reverse_sim

pytestmark = pytest.mark.gpu

FORMS = ["lj", "dexp", "buck", "ljsc", "buff"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def _engine(s, p, x, v, form):
    e = GasEngine(s.n_water, s.n_gas, s.box, form)
    e.set_params(p)
    e.set_state(x, v)
    return e


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def gas120():
    return relaxed_gas(120, 6, 2.6)


@pytest.mark.parametrize("form", FORMS)
def test_forces_vjp_energy_match_oracle(form):
    s, p, x, v = relaxed_gas(80, 5, 2.5, form, seed=2, steps=20)
    e = _engine(s, p, x, v, form)
    pairs = orc.gas_neighbor_pairs(s, x)
    assert _rel(e.forces(), orc.gas_forces(s, p, x, pairs)) < 1e-11
    rng = np.random.default_rng(3)
    w, ac = rng.normal(size=x.shape), rng.normal(size=x.shape)
    F, G, dp = e.force_vjp(w, ac)
    Fo, Go, dpo = orc.gas_forces_grads(s, p, x, w, ac, pairs)
    assert _rel(F, Fo) < 1e-11 and _rel(G, Go) < 1e-10
    assert np.all(np.abs(dp - dpo) <= 1e-10 * np.abs(dpo).max()), (dp, dpo)
    E, dE = e.energy(grads=True)
    Eo, dEo = orc.gas_energy(s, p, x, pairs, grads=True)
    assert abs(E - Eo) <= 1e-11 * abs(Eo)
    assert np.all(np.abs(dE - dEo) <= 1e-10 * np.abs(dEo).max()), (dE, dEo)
    e.close()


def test_forward_follows_the_oracle(gas120):
    s, p, x0, v0 = gas120
    n, nl = 40, 10
    seeds = systems.noise_seeds(n, seed=21)
    xo, vo, lo, sx, sv, gco, outo = orc.gas_forward_sim(s, p, x0, v0, seeds, 1.0, n, nl, 0.001, "diff_ev")
    e = _engine(s, p, x0, v0, "lj")
    loss, parts, centres = e.forward(seeds, 1.0, n, nl, 0.001, "diff_ev")
    xg, vg = e.get_state()
    d = xg - xo
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < 1e-10 and np.abs(vg - vo).max() < 1e-8
    c = centres - gco
    c -= s.box * np.round(c / s.box)
    assert np.abs(c).max() < 1e-10
    assert abs(loss - lo) <= 1e-8 * abs(lo)
    assert np.allclose(parts, outo, rtol=1e-8, atol=0)
    e.close()


@pytest.mark.parametrize("form,loss_type", [("lj", "diff"), ("lj", "diff_ev"), ("buck", "diff"),
                                            ("dexp", "diff_ev"), ("buff", "diff")])
def test_reverse_matches_oracle(form, loss_type):
    """diffusion.jl:1674-1675 on the GPU (reconstruction < 1e-9, |L_rev - L_fwd| < 1e-7) and
    the gradient of the oracle's reverse pass."""
    s, p, x0, v0 = relaxed_gas(80, 5, 2.5, form, seed=4, steps=30)
    n, nl = 40, 10
    seeds = systems.noise_seeds(n, seed=22)
    xf, vf, lfo, sx, sv, gc, _ = orc.gas_forward_sim(s, p, x0, v0, seeds, 1.0, n, nl, 0.001, loss_type)
    _, _, lro, dpo, outo = orc.gas_reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, nl, 0.001, sx, sv, gc,
                                               loss_type)
    e = _engine(s, p, x0, v0, form)
    lf, _, _ = e.forward(seeds, 1.0, n, nl, 0.001, loss_type)
    lr, g, parts = e.reverse(seeds, 1.0, n, nl, nl, 0.001, loss_type)
    xr, _ = e.get_state()
    d = xr - x0
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < 1e-9
    assert abs(lr - lf) < 1e-7 and abs(lr - lro) <= 1e-8 * abs(lro)
    assert np.allclose(parts, outo, rtol=1e-8, atol=0)
    scale = np.abs(dpo * p).max()
    assert np.all(np.abs((g - dpo) * p) <= 1e-7 * scale), (g, dpo)
    e.close()


def test_truncated_reverse_matches_oracle(gas120):
    s, p, x0, v0 = gas120
    n, nl, tr = 60, 20, 7
    seeds = systems.noise_seeds(n, seed=23)
    xf, vf, _, sx, sv, gc, _ = orc.gas_forward_sim(s, p, x0, v0, seeds, 1.0, n, nl, 0.001, "diff")
    xro, _, lro, dpo, _ = orc.gas_reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, tr, 0.001, sx, sv, gc, "diff")
    e = _engine(s, p, x0, v0, "lj")
    e.forward(seeds, 1.0, n, nl, 0.001, "diff")
    lr, g, _ = e.reverse(seeds, 1.0, n, nl, tr, 0.001, "diff")
    xr, _ = e.get_state()
    d = xr - xro
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < 1e-9 and abs(lr - lro) <= 1e-8 * abs(lro)
    scale = np.abs(dpo * p).max()
    assert np.all(np.abs((g - dpo) * p) <= 1e-7 * scale), (g, dpo)
    e.close()


def test_reference_signatures_end_to_end(gas120):
    s, p, x0, v0 = gas120
    n, nl = 40, 10
    seeds = systems.noise_seeds(n, seed=24)
    sys_f, loss_f, acc, grads = forward_sim(x0, v0, seeds, 1.0, n, nl, p, 0.001, 1, "lj", ":diff",
                                            n_gas=s.n_gas, box=s.box)
    assert grads == [None] * len(p) and acc.gas_coords.shape == (4, s.n_gas, 3)
    out = reverse_sim(sys_f.coords, sys_f.velocities, seeds, 1.0, n, nl, nl, p, 0.001, 1,
                      sys_f.loggers, acc, "lj", ":diff")
    sys_r, loss_r, dl_dp, D, l_diff, l_rdf, l_ev = out
    assert abs(loss_r - loss_f) < 1e-7 and D == acc.D and l_diff == loss_r and l_rdf == l_ev == 0.0
    assert np.all(np.isfinite(dl_dp)) and dl_dp.shape == (5,)
    d = sys_r.coords - x0
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < 1e-9
    sys_f.loggers.close()


def test_argument_checks(gas120):
    s, p, x0, v0 = gas120
    e = GasEngine(s.n_water, s.n_gas, s.box)
    with pytest.raises(RevsimError):
        e.forces()                                   # no parameters, no state
    with pytest.raises(RevsimError):
        e.set_params(p[:3])                          # wrong length
    e.set_params(p)
    e.set_state(x0, v0)
    seeds = systems.noise_seeds(20, seed=1)
    with pytest.raises(RevsimError):
        e.reverse(seeds, 1.0, 20, 10, 10, 0.001)     # no forward pass
    with pytest.raises(RevsimError):
        e.forward(seeds, 1.0, 20, 20, 0.001, "diff")  # one loss point: no diffusion coefficient
    e.forward(seeds, 1.0, 20, 10, 0.001, "diff")
    with pytest.raises(RevsimError):
        e.reverse(seeds, 1.0, 20, 5, 5, 0.001)       # differs from the forward pass
    with pytest.raises(RevsimError):
        e.reverse(seeds, 1.0, 20, 10, 10, 0.001, "ev")   # forward recorded no enthalpy term
    with pytest.raises(RevsimError):
        e.forward(seeds, 1.0, 20, 10, 0.001, "diff_rdf_ev")   # no RDF terms set
    with pytest.raises(ValueError):
        e.forward(seeds, 1.0, 20, 10, 0.001, "rdf_diff")
    e.close()


def _rdf_terms(seed):
    """Two squared-error RDF terms (O-O, O-H) with seeded random targets, for the engine and
    for the oracle."""
    from revsim import RdfTerm
    rng = np.random.default_rng(seed)
    spec = [(0, 0, rng.uniform(0, 2, 200)), (0, 1, rng.uniform(0, 2, 200))]
    eng = [RdfTerm(a, b, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, t, 2, 1.0) for a, b, t in spec]
    orl = orc.Loss([orc.RdfTerm(a, b, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, t, 2, 1.0) for a, b, t in spec])
    return eng, orl


@pytest.mark.parametrize("loss_type", ["diff_rdf_ev", "rdf"])
def test_rdf_term_matches_oracle(loss_type):
    """The RDF term of the water atoms (diffusion.jl:759-774, weighted 0.05 / n_blocks) in the
    forward loss and in the reverse gradient, against the oracle."""
    s, p, x0, v0 = relaxed_gas(80, 5, 2.5, "lj", seed=6, steps=30)
    terms, orl = _rdf_terms(7)
    n, nl = 40, 10
    seeds = systems.noise_seeds(n, seed=25)
    xf, vf, lfo, sx, sv, gc, outf = orc.gas_forward_sim(s, p, x0, v0, seeds, 1.0, n, nl, 0.001, loss_type,
                                                        rdf=orl)
    _, _, lro, dpo, outo = orc.gas_reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, nl, 0.001, sx, sv, gc,
                                               loss_type, rdf=orl)
    e = _engine(s, p, x0, v0, "lj")
    e.set_rdf(terms)
    lf, partsf, _ = e.forward(seeds, 1.0, n, nl, 0.001, loss_type)
    assert abs(lf - lfo) <= 1e-9 * abs(lfo) and np.allclose(partsf, outf, rtol=1e-9, atol=0)
    lr, g, parts = e.reverse(seeds, 1.0, n, nl, nl, 0.001, loss_type)
    assert abs(lr - lf) < 1e-7 and np.allclose(parts, outo, rtol=1e-9, atol=0)
    scale = np.abs(dpo * p).max()
    assert np.all(np.abs((g - dpo) * p) <= 1e-7 * scale), (g, dpo)
    e.close()


@pytest.mark.parametrize("form", ["lj", "buck"])
def test_mixed_precision_forces_and_gradient(form):
    """Mixed precision (FP32 pair arithmetic; FP64 state, bonded terms, integrator, adjoints
    and sums) against the FP64 oracle: forces to FP32 rounding, the reconstruction to FP64
    state rounding, the reverse gradient to 1e-3 of its largest component."""
    s, p, x0, v0 = relaxed_gas(80, 5, 2.5, form, seed=4, steps=30)
    e = GasEngine(s.n_water, s.n_gas, s.box, form, precision="mixed")
    e.set_params(p)
    e.set_state(x0, v0)
    assert _rel(e.forces(), orc.gas_forces(s, p, x0)) < 2e-5
    n, nl = 40, 10
    seeds = systems.noise_seeds(n, seed=26)
    xf, vf, lfo, sx, sv, gc, _ = orc.gas_forward_sim(s, p, x0, v0, seeds, 1.0, n, nl, 0.001, "diff_ev")
    _, _, lro, dpo, _ = orc.gas_reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, nl, 0.001, sx, sv, gc, "diff_ev")
    lf, _, _ = e.forward(seeds, 1.0, n, nl, 0.001, "diff_ev")
    lr, g, _ = e.reverse(seeds, 1.0, n, nl, nl, 0.001, "diff_ev")
    xr, _ = e.get_state()
    d = xr - x0
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < 1e-6 and abs(lr - lf) < 1e-7
    assert abs(lf - lfo) <= 1e-3 * abs(lfo)
    scale = np.abs(dpo * p).max()
    assert np.all(np.abs((g - dpo) * p) <= 1e-3 * scale), (g, dpo)
    e.close()
