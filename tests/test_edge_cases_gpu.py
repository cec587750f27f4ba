"""Edge cases of the water engine on the GPU: a run of zero steps; a replica of one molecule
(no pair terms at all) batched with a liquid box; the enthalpy term with replicas of uneven
size; the learned term switched on with the barostat; calls in the wrong order."""

import numpy as np
import pytest

from conftest import relaxed_water
from oracle import orc
from revsim import Engine, RevsimError, constants as C, mlp, systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def _engine(n_mol, box, prec="fp64", **kw):
    e = Engine(n_mol, box, precision=prec, **kw)
    e.set_params(C.default_params())
    return e


def test_zero_steps(small_water):
    n_mol, box, x, v = small_water
    e = _engine(n_mol, box)
    e.set_enth_vap(True)
    e.set_state(x, v)
    loss = e.forward(np.zeros(0, dtype=np.uint64), 1.0, 0, 1, 0.001)
    xg, vg = e.get_state()
    assert np.array_equal(xg, x) and np.array_equal(vg, v) and loss[0] == 0.0
    with pytest.raises(RevsimError):
        e.reverse(np.zeros(0, dtype=np.uint64), 1.0, 0, 1, 1, 0.001)
    e.close()


def test_single_molecule_replica_next_to_a_liquid_box(small_water):
    """A lone molecule has no pair terms: its forces are its bonds and angle, its RDF is empty
    and its gradient comes from the bonded parameters only; batching it with a liquid box
    changes nothing for either."""
    n_mol, box, x, v = small_water
    x1, v1 = x[:3].copy(), v[:3].copy()
    n = 20
    seeds = np.stack([systems.noise_seeds(n, seed=6), systems.noise_seeds(n, seed=7)], axis=1)
    eb = _engine([1, n_mol], [box, box])
    eb.set_enth_vap(True)
    eb.set_state(np.concatenate([x1, x]), np.concatenate([v1, v]))
    F = eb.forces()
    lfb = eb.forward(seeds, 1.0, n, n, 0.001)
    lrb, gb = eb.reverse(seeds, 1.0, n, n, n, 0.001)
    eb.close()
    s1 = orc.make_system(1, box)
    Fo = orc.forces(s1, C.default_params(), x1, np.zeros((0, 2), dtype=np.int32))
    assert np.linalg.norm(F[:3] - Fo) <= 1e-10 * np.linalg.norm(Fo)
    assert np.all(np.isfinite(gb)) and np.all(gb[0, :3] == 0.0)   # no LJ / charge terms
    for r, (xr, vr, nm) in enumerate([(x1, v1, 1), (x, v, n_mol)]):
        e = _engine(nm, box)
        e.set_enth_vap(True)
        e.set_state(xr, vr)
        lf = e.forward(seeds[:, r], 1.0, n, n, 0.001)
        lr, g = e.reverse(seeds[:, r], 1.0, n, n, n, 0.001)
        e.close()
        assert abs(lf[0] - lfb[r]) <= 1e-12 * abs(lf[0]) and abs(lr[0] - lrb[r]) <= 1e-12 * abs(lr[0])
        assert np.abs(g[0] - gb[r]).max() <= 1e-10 * np.abs(g[0]).max()


def test_barostat_with_the_learned_term(small_water):
    """The barostat's energies include the learned pair correction: the FP64 engine follows
    the oracle's barostatted run with it switched on."""
    n_mol, box, x, v = small_water
    th = mlp.init_params(3) + np.random.default_rng(4).normal(scale=0.01, size=mlp.N_PARAMS)
    p = np.concatenate([C.default_params(), th])
    seeds = systems.noise_seeds(60, seed=12)
    s = orc.make_system(n_mol, box, mlp=True)
    b = orc.make_barostat(box, seed=3, n_steps=6)
    xo, _ = orc.forward_sim_barostat(s, p, x, v, seeds, 1.0, 60, 0.001, b)
    e = Engine(n_mol, box, precision="fp64", mlp=True)
    e.set_params(p)
    e.set_state(x, v)
    e.set_barostat(True, n_steps=6, seed=3)
    e.forward(seeds, 1.0, 60, 60, 0.001, calc_loss=False)
    bx, _, na, nacc = e.barostat_state()
    xg, _ = e.get_state()
    e.close()
    assert na[0] == b.n_draws and nacc[0] == b.n_accepted_total and nacc[0] > 0
    assert abs(bx[0] - s.box) <= 1e-12 * s.box
    d = xg - xo
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() <= 1e-9


def test_calls_in_the_wrong_order(small_water):
    n_mol, box, x, v = small_water
    e = Engine(n_mol, box, precision="fp64")
    with pytest.raises(RevsimError):
        e.forces()                      # no parameters, no state
    e.set_params(C.default_params())
    with pytest.raises(RevsimError):
        e.loss_and_grads()              # no state
    e.set_state(x, v)
    with pytest.raises(RevsimError):    # no loss set
        e.forward(systems.noise_seeds(4), 1.0, 4, 4, 0.001)
        e.reverse(systems.noise_seeds(4), 1.0, 4, 4, 4, 0.001)
    with pytest.raises(RevsimError):
        e.set_params(np.ones(3))        # wrong length
    with pytest.raises(RevsimError):
        e.set_barostat(True, n_steps=0)
    e.close()
