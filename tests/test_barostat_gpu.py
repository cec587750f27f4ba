"""The engine's Monte-Carlo barostat (revsim_set_barostat; MonteCarloBarostatNoUnits,
water.jl:789-865) against the FP64 oracle's barostatted forward run (orc_forward_sim_barostat)
on the same seeded inputs: the same moves accepted, the final box to 1e-12 and the positions
to 1e-9 nm (FP64 mode); batched replicas equal to single runs; the barostat's step count
carried across forward calls; forward_sim(use_barostat=True) through the reference
signature; a barostatted forward pass refused as a reverse record; revsim_set_box.
"""

import numpy as np
import pytest

from conftest import relaxed_water
from oracle import orc
from revsim import Engine, RevsimError, constants as C, systems
from revsim.water import forward_sim

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def _min_image(d, box):
    return d - box * np.round(d / box)


@pytest.mark.parametrize("n_baro", [5, 7])
def test_barostatted_run_matches_oracle(small_water, n_baro):
    n_mol, box, x, v = small_water
    p = np.array(C.default_params())
    n = 120
    seeds = systems.noise_seeds(n, seed=3)
    s = orc.make_system(n_mol, box)
    b = orc.make_barostat(box, seed=7, n_steps=n_baro)
    xo, vo = orc.forward_sim_barostat(s, p, x, v, seeds, 1.0, n, 0.001, b)
    e = Engine(n_mol, box, precision="fp64")
    e.set_params(p)
    e.set_state(x, v)
    e.set_barostat(True, n_steps=n_baro, seed=7)
    e.forward(seeds, 1.0, n, n, 0.001, calc_loss=False)
    xg, vg = e.get_state()
    bx, vs, na, nacc = e.barostat_state()
    e.close()
    assert na[0] == b.n_draws == n // n_baro
    assert nacc[0] == b.n_accepted_total and nacc[0] > 3
    assert abs(bx[0] - s.box) <= 1e-12 * s.box and bx[0] != box
    assert abs(vs[0] - b.volume_scale) <= 1e-12 * b.volume_scale
    assert np.abs(_min_image(xg - xo, s.box)).max() <= 1e-9
    assert np.abs(vg - vo).max() <= 1e-7


def test_batched_replicas_equal_single_runs():
    sizes, boxes = [150, 120], [2.6, 2.45]
    xs, vs = zip(*[relaxed_water(m, b_, seed=60 + i, steps=30) for i, (m, b_) in enumerate(zip(sizes, boxes))])
    p = np.array(C.default_params())
    n = 90
    seeds = np.stack([systems.noise_seeds(n, seed=90 + r) for r in range(2)], axis=1)
    eb = Engine(sizes, boxes, precision="fp64")
    eb.set_params(p)
    eb.set_state(np.concatenate(xs), np.concatenate(vs))
    eb.set_barostat(True, n_steps=6, seed=11)
    eb.forward(seeds, 1.0, n, n, 0.001, calc_loss=False)
    xb, _ = eb.get_state()
    bb, _, nab, naccb = eb.barostat_state()
    eb.close()
    off = 0
    for r in range(2):
        e = Engine(sizes[r], boxes[r], precision="fp64")
        e.set_params(p)
        e.set_state(xs[r], vs[r])
        e.set_barostat(True, n_steps=6, seed=11 + r)   # replica r draws from seed + r
        e.forward(seeds[:, r], 1.0, n, n, 0.001, calc_loss=False)
        x1, _ = e.get_state()
        b1, _, na1, nacc1 = e.barostat_state()
        e.close()
        assert na1[0] == nab[r] and nacc1[0] == naccb[r] and b1[0] == bb[r]
        assert np.abs(x1 - xb[off:off + 3 * sizes[r]]).max() <= 1e-12
        off += 3 * sizes[r]


def test_step_count_carries_across_forward_calls(small_water):
    """Two forward calls of 60 steps attempt at the same steps as one call of 120."""
    n_mol, box, x, v = small_water
    p = np.array(C.default_params())
    seeds = systems.noise_seeds(120, seed=5)
    out = []
    for split in (False, True):
        e = Engine(n_mol, box, precision="fp64")
        e.set_params(p)
        e.set_state(x, v)
        e.set_barostat(True, n_steps=7, seed=2)
        if split:
            e.forward(seeds[:60], 1.0, 60, 60, 0.001, calc_loss=False)
            e.forward(seeds[60:], 1.0, 60, 60, 0.001, calc_loss=False)
        else:
            e.forward(seeds, 1.0, 120, 120, 0.001, calc_loss=False)
        out.append((e.get_state()[0], e.barostat_state()))
        e.close()
    assert out[0][1][2][0] == out[1][1][2][0] == 120 // 7
    assert out[0][1][0][0] == out[1][1][0][0]
    assert np.abs(_min_image(out[0][0] - out[1][0], out[0][1][0][0])).max() <= 1e-12


def test_reference_signature_and_reverse_refusal(small_water):
    n_mol, box, x, v = small_water
    p = np.array(C.default_params())
    seeds = systems.noise_seeds(90, seed=8)
    sys_f, _, _ = forward_sim(x, v, box, seeds, 1.0, 90, 90, p, 0.001, 1, "lj", "rdf",
                              calc_loss=False, use_barostat=True, precision="mixed")
    eng = sys_f.engine
    assert sys_f.boundary != box and abs(sys_f.boundary - box) < 0.1 * box
    with pytest.raises(RevsimError):   # an equilibration run leaves no reverse record
        eng.set_loss([])
        eng.set_enth_vap(True)
        eng.reverse(seeds, 1.0, 90, 90, 90, 0.001)
    # the next run starts from the equilibrated state in the equilibrated box
    sys2, loss, _ = forward_sim(sys_f.coords, sys_f.velocities, sys_f.boundary, seeds[:20], 1.0, 20, 20,
                                p, 0.001, 1, "lj", "enth_vap", engine=eng)
    assert sys2.boundary == sys_f.boundary and np.isfinite(loss)
    eng.close()


def test_set_box(small_water):
    n_mol, box, x, v = small_water
    e = Engine(n_mol, box, precision="fp64")
    e.set_params(C.default_params())
    e.set_box(2.7)
    e.set_state(x, v)
    F = e.forces()
    s = orc.make_system(n_mol, 2.7)
    Fo = orc.forces(s, C.default_params(), x, orc.neighbor_pairs(s, x))
    assert np.linalg.norm(F - Fo) <= 1e-10 * np.linalg.norm(Fo)
    with pytest.raises(RevsimError):
        e.set_box(2.0)   # below twice the 1.2 nm neighbour cutoff
    e.close()
