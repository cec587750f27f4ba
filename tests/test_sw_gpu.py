"""Stillinger-Weber diamond engine (librevsim.so, include/revsim_sw.h) against the FP64 CPU
oracle (oracle/sw_oracle.c) on the same seeded inputs.

Bars: the active pair set bit-exact; forces, stress and every derivative within 1e-10
relative in FP64 mode and 1e-5 (forces) / 1e-4 (gradients) in mixed mode; the reference's
self-check (diamond.jl:1910-1942: 12 steps, loss every 5, truncation 12, gamma 4/ps,
dt 0.5 fs) reproduced, and the reverse-pass gradient equal to the oracle's.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRECS = [("fp64", 1e-10, 1e-9), ("mixed", 1e-5, 1e-4)]


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def _crystal(cells=3, noise=0.01, seed=4, vseed=5):
    from revsim import diamond as D
    x, box = D.diamond_coords(cells, noise=noise, seed=seed)
    v = D.mb_velocities(len(x), seed=vseed)
    return x, v, box


def _engine(x, v, box, prec="fp64", **kw):
    from revsim import SwEngine, diamond as D
    e = SwEngine(len(x), box, precision=prec, **kw)
    e.set_params(D.default_params())
    e.set_state(x, v)
    return e


def nrel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.mark.parametrize("cells,noise", [(3, 0.01), (5, 0.005)])
def test_active_pairs_bit_exact(cells, noise):
    from oracle import orc
    from revsim import diamond as D
    x, v, box = _crystal(cells, noise)
    s = orc.make_sw_system(len(x), box)
    ref = orc.sw_pairs(s, D.default_params(), x)
    for prec in ("fp64", "mixed"):
        with _engine(x, v, box, prec) as e:
            got = e.active_pairs()
        assert np.array_equal(got, ref)


@pytest.mark.parametrize("prec,ftol,gtol", PRECS)
def test_forces(prec, ftol, gtol):
    from oracle import orc
    from revsim import diamond as D
    x, v, box = _crystal()
    s = orc.make_sw_system(len(x), box)
    F_ref = orc.sw_forces(s, D.default_params(), x)
    with _engine(x, v, box, prec) as e:
        F = e.forces()
    assert nrel(F, F_ref) <= ftol


@pytest.mark.parametrize("prec,ftol,gtol", PRECS)
def test_force_vjp_and_parameter_contraction(prec, ftol, gtol):
    from oracle import orc
    from revsim import diamond as D
    x, v, box = _crystal()
    rng = np.random.default_rng(7)
    w = rng.normal(size=x.shape)
    ac = rng.normal(size=x.shape)
    s = orc.make_sw_system(len(x), box)
    F_ref, G_ref, J = orc.sw_forces_grads(s, D.default_params(), x, w)
    dth_ref = (ac.reshape(-1)[:, None] * J).sum(axis=0)
    with _engine(x, v, box, prec) as e:
        F, G, dth = e.force_vjp(w, ac)
    assert nrel(F, F_ref) <= ftol
    assert nrel(G, G_ref) <= gtol
    assert np.abs(dth[0] - dth_ref).max() <= gtol * np.abs(dth_ref).max()


def test_forces_deterministic_and_lane_independent():
    x, v, box = _crystal(5, 0.005)
    with _engine(x, v, box, "mixed") as e:
        F1 = e.forces()
        F2 = e.forces()
        e.set_lanes(32)
        F3 = e.forces()
    assert np.array_equal(F1, F2)
    assert np.array_equal(F1, F3)


def test_noise_matches_oracle():
    from oracle import orc
    x, v, box = _crystal()
    s = orc.make_sw_system(len(x), box)
    with _engine(x, v, box) as e:
        xi = e.noise(123456789)
    ref = orc.sw_noise(s, 123456789)
    assert np.abs(xi - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("prec,ftol,gtol", PRECS)
def test_stress_and_loss_gradients(prec, ftol, gtol):
    from oracle import orc
    from revsim import diamond as D
    x, v, box = _crystal()
    rng = np.random.default_rng(3)
    target = rng.normal(scale=50.0, size=9)
    s = orc.make_sw_system(len(x), box)
    p = D.default_params()
    sig_ref = orc.sw_stress(s, p, x, v)
    L = orc.make_sw_loss(D.STRESS_WEIGHT, target)
    l_ref, gx_ref, gv_ref, gp_ref = orc.sw_loss_grad(s, p, L, x, v)
    with _engine(x, v, box, prec) as e:
        sig = e.stress()[0]
        e.set_loss(D.STRESS_WEIGHT, target)
        l, gx, gv, gp = e.loss_grad()
    assert nrel(sig, sig_ref) <= ftol
    assert abs(l[0] - l_ref) <= gtol * abs(l_ref)
    assert nrel(gx, gx_ref) <= gtol
    assert nrel(gv, gv_ref) <= gtol
    assert np.abs(gp[0] - gp_ref).max() <= gtol * np.abs(gp_ref).max()


def test_forward_trajectory_matches_oracle():
    from oracle import orc
    from revsim import diamond as D
    x, v, box = _crystal(3, 0.003)
    seeds = np.arange(1, 13, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    s = orc.make_sw_system(len(x), box)
    L = orc.make_sw_loss(D.STRESS_WEIGHT)
    xf, vf, lf, _, _ = orc.sw_forward_sim(s, D.default_params(), x, v, seeds, 4.0, 12, 5, 0.0005, L)
    with _engine(x, v, box, "fp64") as e:
        e.set_loss()
        loss, nb = e.forward(seeds, 4.0, 12, 5, 0.0005)
        xg, vg = e.get_state()
    assert nb == 3
    d = xg - xf
    d -= np.round(d / box) * box
    assert np.abs(d).max() <= 1e-11
    assert np.abs(vg - vf).max() <= 1e-9 * np.abs(vf).max()
    assert abs(loss[0] - lf) <= 1e-9 * abs(lf)


@pytest.mark.parametrize("prec,ftol,gtol", PRECS)
@pytest.mark.parametrize("trunc", [12, 3])
def test_reverse_selfcheck_and_gradient(prec, ftol, gtol, trunc):
    """diamond.jl:1939-1941: the start state is rebuilt (truncation 12 reaches step 0) and
    the reverse loss equals the forward loss; the gradient equals the oracle's."""
    from oracle import orc
    from revsim import diamond as D
    x, v, box = _crystal(3, 0.003)
    seeds = np.arange(1, 13, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    s = orc.make_sw_system(len(x), box)
    L = orc.make_sw_loss(D.STRESS_WEIGHT)
    p = D.default_params()
    xf, vf, lf, sx, sv = orc.sw_forward_sim(s, p, x, v, seeds, 4.0, 12, 5, 0.0005, L)
    _, _, lr_ref, g_ref = orc.sw_reverse_sim(s, p, xf, vf, seeds, 4.0, 12, 5, trunc, 0.0005, sx, sv, L)
    with _engine(x, v, box, prec) as e:
        e.set_loss()
        lfw, nb = e.forward(seeds, 4.0, 12, 5, 0.0005)
        lrv, g = e.reverse(seeds, 4.0, 12, 5, trunc, 0.0005)
        xr, vr = e.get_state()
    assert abs(lrv[0] - lfw[0]) <= 1e-12 * abs(lfw[0])
    assert abs(lrv[0] - lr_ref) <= gtol * abs(lr_ref)
    assert np.abs(g[0] - g_ref).max() <= gtol * np.abs(g_ref).max(), (g[0], g_ref)
    if trunc == 12:
        d = xr - x
        d -= np.round(d / box) * box
        assert np.abs(d).max() < (1e-8 if prec == "fp64" else 1e-6)


def test_batched_replicas_equal_single_runs():
    from revsim import SwEngine, diamond as D
    systems = [_crystal(3, 0.003, seed=11), _crystal(4, 0.002, seed=12), _crystal(3, 0.003, seed=13)]
    temps = [280.0, 300.0, 320.0]
    seeds = np.arange(1, 21, dtype=np.uint64).reshape(20, 1) * np.uint64(0x2545F4914F6CDD1D) + \
        np.arange(3, dtype=np.uint64).reshape(1, 3)
    singles = []
    for r, (x, v, box) in enumerate(systems):
        with _engine(x, v, box, "mixed", temp=temps[r]) as e:
            e.set_loss()
            lf, _ = e.forward(seeds[:, r], 1.0, 20, 10, 0.0005)
            lr, g = e.reverse(seeds[:, r], 1.0, 20, 10, 10, 0.0005)
            singles.append((lf[0], lr[0], g[0]))
    eb = SwEngine([len(s[0]) for s in systems], [s[2] for s in systems], temp=temps, precision="mixed")
    eb.set_params(D.default_params())
    eb.set_state(np.concatenate([s[0] for s in systems]), np.concatenate([s[1] for s in systems]))
    eb.set_loss()
    lf, _ = eb.forward(seeds, 1.0, 20, 10, 0.0005)
    lr, g = eb.reverse(seeds, 1.0, 20, 10, 10, 0.0005)
    eb.close()
    for r in range(3):
        assert abs(lf[r] - singles[r][0]) <= 1e-12 * abs(singles[r][0])
        assert abs(lr[r] - singles[r][1]) <= 1e-12 * abs(singles[r][1])
        assert np.abs(g[r] - singles[r][2]).max() <= 1e-12 * np.abs(singles[r][2]).max()


def test_reference_entry_points():
    """forward_sim / reverse_sim with the argument order of diamond.jl:1394 and 1757."""
    from revsim import diamond as D
    from revsim import sw
    x, v, box = _crystal(3, 0.003)
    seeds = np.arange(1, 13, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    p = D.default_params()
    sys_f, loss_f, acc, logs, _, _ = sw.forward_sim(x, v, seeds, 4.0, 12, 5, 0, p, None, 0.0005,
                                                     box=box, precision="fp64")
    sys_r, loss_r, g, _ = sw.reverse_sim(sys_f.coords, sys_f.velocities, seeds, 4.0, 12, 5, 12, 0,
                                         p, None, 0.0005, 1, sys_f.loggers, acc)
    assert acc["n_blocks"] == 3
    assert abs(loss_r - loss_f) <= 1e-12 * abs(loss_f)
    assert g.shape == (7,) and np.all(np.isfinite(g))
    sys_f.loggers.close()


def test_errors():
    from revsim import RevsimError, SwEngine, diamond as D
    x, v, box = _crystal()
    with pytest.raises(RevsimError):   # box below 3 cells of a sigma + skin
        SwEngine(len(x), 0.8).set_params(D.default_params())
    with _engine(x, v, box) as e:
        with pytest.raises(RevsimError):   # loss not set
            e.loss_grad()
        e.set_loss()
        with pytest.raises(RevsimError):   # no forward record
            e.reverse(np.ones(4, dtype=np.uint64), 1.0, 4, 2, 2, 0.0005)
        with pytest.raises(RevsimError):
            e.set_params(np.ones(6))


def test_hot_start_rebuilds_more_often_with_the_same_result():
    """0.01 nm noise makes atoms move more than skin / 2 within 10 steps; the call is rerun
    with shorter rebuild intervals and returns what an every-step rebuild gives."""
    x, v, box = _crystal(3, 0.01)
    seeds = np.arange(1, 21, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    out = []
    for nf in (10, 1):
        with _engine(x, v, box, "mixed", n_steps_nf=nf) as e:
            e.set_loss()
            lf, _ = e.forward(seeds, 4.0, 20, 10, 0.0005)
            xg, vg = e.get_state()
            out.append((lf, xg, vg))
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
    assert np.array_equal(out[0][0], out[1][0])
