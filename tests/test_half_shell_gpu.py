"""Half-shell pair evaluation (revsim_set_pair_mode REVSIM_PAIRS_HALF_SHELL): each molecule
pair evaluated once by its owner, the partner's share gathered by a second kernel.

* forces, force VJP and the dtheta contraction on the tip3p.pdb box (3.0 nm) against the FP64
  oracle at the mixed-precision bars (1e-5 / 1e-4), for every trained parameter set, and
  against the both-sides kernels of the same handle (1e-5: the same FP32 pair arithmetic
  summed in another order);
* the learned pair correction (coefficient adjoints taken once per pair) and the buffered
  14-7 form against the oracle at the mixed bars;
* a 20-step gradient (gamma = 1/ps) against the oracle at the mixed bar (1e-4, 3e-4 for the
  exponential forms), on the tip3p box and on a 4.5 nm box of 3,000 molecules;
* with the exactly reversible integrator the reverse pass rebuilds 1,000 steps at gamma = 0 bit
  for bit (forward and reverse forces are the same bits), as with the both-sides kernels;
* CUDA-graph replay gives the same bits as plain launches;
* the mode is refused for FP64 handles, not in effect in boxes too small for one periodic image
  per molecule pair, and a mode change between the forward and the reverse pass is refused.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import Engine, RdfTerm, RevsimError, constants as C, systems

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


def _term(s, x):
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    return (orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)]),
            [RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])


@pytest.mark.parametrize("name", SETS)
def test_forces_and_vjp_match_the_oracle_and_both_sides(name):
    x, box, sets = load()
    form, p = sets[name]
    rng = np.random.default_rng(17)
    w, ac = rng.normal(size=x.shape), rng.normal(size=x.shape)
    s = orc.make_system(895, box, form)
    Fo, Go, J = orc.forces_grads(s, p, x, orc.neighbor_pairs(s, x), w)
    out = {}
    for mode in ("both_sides", "half_shell"):
        e = Engine(895, box, inter_type=form, precision="mixed")
        e.set_params(p)
        e.set_pair_mode(mode)
        assert e.pair_mode()[1] == mode
        e.set_state(x, np.zeros_like(x))
        out[mode] = (e.forces(),) + e.force_vjp(w, ac)
        e.close()
    F0, F, G, th = out["half_shell"]
    assert nrel(F0, Fo) < 1e-5
    assert nrel(F, Fo) < 1e-5
    assert nrel(G, Go) < 1e-4
    assert np.all(scaled_err(th[0], ac.ravel() @ J, p) < 1e-4)
    Fb, _, Gb, thb = out["both_sides"]
    assert nrel(F, Fb) < 1e-5
    assert nrel(G, Gb) < 1e-4
    assert np.all(scaled_err(th[0], thb[0], p) < 1e-4)


def _gradient_vs_oracle(n_mol, box, x, v, form, p, n=20):
    s = orc.make_system(n_mol, box, form)
    ol, terms = _term(s, x)
    seeds = systems.noise_seeds(n, seed=4)
    xf, vf, lfo, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, ol)
    _, _, _, go = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, ol)
    e = Engine(n_mol, box, inter_type=form, precision="mixed")
    e.set_params(p)
    e.set_loss(terms)
    e.set_pair_mode("half_shell")
    assert e.pair_mode()[1] == "half_shell"
    e.set_state(x, v)
    lf = e.forward(seeds, 1.0, n, n, 0.001)
    _, g = e.reverse(seeds, 1.0, n, n, n, 0.001)
    e.close()
    assert abs(lf[0] - lfo) < 1e-5 * abs(lfo)
    return scaled_err(g[0], go, p)


@pytest.mark.parametrize("name", SETS)
def test_tip3p_gradient_matches_the_oracle(name):
    x, box, sets = load()
    form, p = sets[name]
    v = systems.mb_velocities(895, seed=3)
    err = _gradient_vs_oracle(895, box, x, v, form, p)
    assert np.all(err < (1e-4 if form == "lj" else 3e-4)), err


def test_box45_gradient_matches_the_oracle():
    from conftest import relaxed_water
    x, v = relaxed_water(3000, 4.5, seed=9, steps=20)
    err = _gradient_vs_oracle(3000, 4.5, x, v, "lj", np.array(C.default_params("lj")), n=10)
    assert np.all(err < 1e-4), err


def test_exact_reversal_is_bit_exact(cfg1_water):
    n_mol, box, x, v = cfg1_water
    s = orc.make_system(n_mol, box)
    _, terms = _term(s, x)
    e = Engine(n_mol, box, precision="mixed")
    e.set_params(C.default_params())
    e.set_loss(terms)
    e.set_integrator("exact")
    e.set_pair_mode("half_shell")
    e.set_state(x, v)
    e.autotune()
    e.set_state(x, v)
    n = 1000
    seeds = systems.noise_seeds(n, seed=3)
    e.forward(seeds, 0.0, n, n, 0.001)
    x1, v1 = e.get_state()
    e.reverse(seeds, 0.0, n, n, n, 0.001)
    x0, v0 = e.get_state()
    # the forward pass started from the state on the 2^-48 grid
    L = np.rint(box * 2.0 ** 48) * 2.0 ** -48
    xq = np.rint(x * 2.0 ** 48) * 2.0 ** -48
    xq = xq - np.floor(xq / L) * L
    xq = np.where(xq < 0, xq + L, np.where(xq >= L, xq - L, xq))
    np.testing.assert_array_equal(x0, xq)
    np.testing.assert_array_equal(v0, np.rint(v * 2.0 ** 48) * 2.0 ** -48)
    assert not np.array_equal(x1, x0)


def test_graph_replay_is_bit_identical(cfg1_water):
    n_mol, box, x, v = cfg1_water
    s = orc.make_system(n_mol, box)
    _, terms = _term(s, x)
    seeds = systems.noise_seeds(60, seed=8)
    out = []
    for graph in (False, True):
        e = Engine(n_mol, box, precision="mixed")
        e.set_params(C.default_params())
        e.set_loss(terms)
        e.set_pair_mode("half_shell")
        e.set_graph_mode(graph)
        for _ in range(2):
            e.set_state(x, v)
            e.forward(seeds, 1.0, 60, 30, 0.001)
            xf, vf = e.get_state()
            lr, g = e.reverse(seeds, 1.0, 60, 30, 30, 0.001)
        out.append((xf, vf, lr, g))
        e.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    np.testing.assert_allclose(out[0][3], out[1][3], rtol=1e-12, atol=0)


def test_mode_rules():
    x, box, sets = load()
    e64 = Engine(895, box, precision="fp64")
    with pytest.raises(RevsimError):
        e64.set_pair_mode("half_shell")
    e64.close()
    # 2.48 nm: below 2 (cutoff + 0.3) + 0.02 nm, so the both-sides kernels run
    small = Engine(400, 2.48, precision="mixed")
    small.set_pair_mode("half_shell")
    assert small.pair_mode() == ("half_shell", "both_sides")
    small.close()
    e = Engine(895, box, precision="mixed")
    e.set_params(sets["tip3p"][1])
    s = orc.make_system(895, box)
    _, terms = _term(s, x)
    e.set_loss(terms)
    e.set_state(x, systems.mb_velocities(895, seed=3))
    seeds = systems.noise_seeds(10, seed=2)
    e.forward(seeds, 1.0, 10, 10, 0.001)
    e.set_pair_mode("half_shell")
    with pytest.raises(RevsimError):
        e.reverse(seeds, 1.0, 10, 10, 10, 0.001)
    e.close()


def _mlp_theta(scale):
    from revsim import mlp
    th = mlp.init_params(3) + np.random.default_rng(4).normal(scale=scale, size=mlp.N_PARAMS)
    return np.concatenate([C.default_params("lj"), th])


def test_learned_term_forces_vjp_and_contraction(cfg1_water):
    """The learned pair correction in the owner kernel: its coefficient adjoints are taken
    once per pair against ca_a - ca_b.  Forces, VJP and the contraction over all 15,946
    parameters against the FP64 oracle at the mixed bars, and against the both-sides
    kernels of the same handle."""
    n_mol, box, x, v = cfg1_water
    theta = _mlp_theta(0.05)
    rng = np.random.default_rng(7)
    w, ac = rng.normal(size=x.shape), rng.normal(size=x.shape)
    s = orc.make_system(n_mol, box, "lj", mlp=True)
    pairs = orc.neighbor_pairs(s, x)
    Fo, Go, _ = orc.forces_grads(s, theta, x, pairs, w, jac=False)
    tho = orc.contract(s, theta, x, pairs, ac)
    out = {}
    for mode in ("both_sides", "half_shell"):
        e = Engine(n_mol, box, inter_type="lj", precision="mixed", mlp=True)
        e.set_params(theta)
        e.set_pair_mode(mode)
        assert e.pair_mode()[1] == mode
        e.set_state(x, v)
        out[mode] = e.force_vjp(w, ac)
        e.close()
    F, G, th = out["half_shell"]
    assert nrel(F, Fo) < 1e-5
    assert nrel(G, Go) < 1e-4
    cl = slice(0, 7)
    sc = np.abs(tho[cl] * theta[cl])
    assert np.all(np.abs((th[0][cl] - tho[cl]) * theta[cl]) / np.maximum(sc, 0.01 * sc.max()) < 1e-4)
    assert np.abs(th[0][7:] - tho[7:]).max() < 1e-4 * np.abs(tho[7:]).max()
    Fb, Gb, thb = out["both_sides"]
    assert nrel(F, Fb) < 1e-5
    assert np.abs(th[0][7:] - thb[0][7:]).max() < 1e-4 * np.abs(thb[0][7:]).max()


def test_buffered_14_7_forces(cfg1_water):
    """The buffered 14-7 pair form (not among the trained parameter sets) in the owner
    kernel: forces and VJP against the oracle."""
    n_mol, box, x, v = cfg1_water
    p = np.array(C.default_params("buff"))
    rng = np.random.default_rng(9)
    w, ac = rng.normal(size=x.shape), rng.normal(size=x.shape)
    s = orc.make_system(n_mol, box, "buff")
    Fo, Go, J = orc.forces_grads(s, p, x, orc.neighbor_pairs(s, x), w)
    e = Engine(n_mol, box, inter_type="buff", precision="mixed")
    e.set_params(p)
    e.set_pair_mode("half_shell")
    assert e.pair_mode()[1] == "half_shell"
    e.set_state(x, v)
    F, G, th = e.force_vjp(w, ac)
    e.close()
    assert nrel(F, Fo) < 1e-5
    assert nrel(G, Go) < 1e-4
    assert np.all(scaled_err(th[0], ac.ravel() @ J, p) < 1e-4)
