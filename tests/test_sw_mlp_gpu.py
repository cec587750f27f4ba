"""The learned radial term of the Stillinger-Weber engine (revsim_sw_desc.mlp) against the
FP64 oracle (sw_oracle.c with orc_sw_system.mlp).

Bars: forces and the stress 1e-10 (FP64) / 1e-5 (mixed) relative; the VJP, the parameter
contraction and the stress-loss gradients 1e-9 (FP64) / 1e-4 (mixed) relative to the
largest entry of each parameter group (the 7 SW parameters; each MLP layer); the reverse
pass of the reference's self-check run (diamond.jl:1910-1942) against the oracle's gradient
1e-6 (FP64) / 1e-4 (mixed) per group; zero MLP weights give the plain SW engine; batched
replicas give each replica its own MLP gradient; the reference signature maps params_gnn to
the MLP parameters.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import SwEngine, diamond as D, mlp

pytestmark = pytest.mark.gpu

PRECS = [("fp64", 1e-10, 1e-9), ("mixed", 1e-5, 1e-4)]


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


@pytest.fixture(scope="module")
def theta():
    """SW parameters and a strongly-on learned term: one MLP type perturbed by N(0, 0.1) with
    its output layer (w3, b3) scaled by 30, so that the term moves the forces by ~0.2 %
    (the SW pair energies are ~1e3 kJ/mol)."""
    th = D.init_mlp_params(3) + np.random.default_rng(8).normal(scale=0.1, size=D.MLP_NPARAMS)
    th[D.MLP_NPARAMS - 65:] *= 30.0
    return np.concatenate([D.default_params(), th])


def _crystal(cells=3, noise=0.01, seed=4, vseed=5):
    x, box = D.diamond_coords(cells, noise=noise, seed=seed)
    return x, D.mb_velocities(len(x), seed=vseed), box


def _engine(x, v, box, prec, theta, **kw):
    e = SwEngine(len(x), box, precision=prec, mlp=True, **kw)
    assert e.n_params == 7 + D.MLP_NPARAMS
    e.set_params(theta)
    e.set_state(x, v)
    return e


def nrel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def groups():
    """SW parameters, then W1+b1, W2+b2, w3+b3 of the MLP."""
    a = mlp.H * mlp.NRBF + mlp.H
    b = a + mlp.H * mlp.H + mlp.H
    return [np.arange(7), 7 + np.arange(a), 7 + np.arange(a, b), 7 + np.arange(b, D.MLP_NPARAMS)]


def group_err(g, ref):
    return max(float(np.abs(g[ix] - ref[ix]).max() / np.abs(ref[ix]).max()) for ix in groups())


@pytest.mark.parametrize("prec,ftol,gtol", PRECS)
def test_forces_vjp_and_contraction(theta, prec, ftol, gtol):
    x, v, box = _crystal()
    rng = np.random.default_rng(7)
    w, ac = rng.normal(size=x.shape), rng.normal(size=x.shape)
    s = orc.make_sw_system(len(x), box, mlp=True)
    F_ref, G_ref, _ = orc.sw_forces_grads(s, theta, x, w, jac=False)
    dth_ref = orc.sw_contract(s, theta, x, ac)
    F0 = orc.sw_forces(orc.make_sw_system(len(x), box), theta[:7], x)
    assert nrel(F_ref, F0) > 1e-3                  # the learned term is on
    with _engine(x, v, box, prec, theta) as e:
        F2 = e.forces()
        F, G, dth = e.force_vjp(w, ac)
    assert nrel(F, F_ref) <= ftol and np.array_equal(F, F2)
    assert nrel(G, G_ref) <= gtol
    assert group_err(dth[0], dth_ref) <= gtol, group_err(dth[0], dth_ref)


@pytest.mark.parametrize("prec,ftol,gtol", PRECS)
def test_stress_and_loss_gradients(theta, prec, ftol, gtol):
    x, v, box = _crystal()
    target = np.random.default_rng(3).normal(scale=50.0, size=9)
    s = orc.make_sw_system(len(x), box, mlp=True)
    sig_ref = orc.sw_stress(s, theta, x, v)
    l_ref, gx_ref, gv_ref, gp_ref = orc.sw_loss_grad(s, theta, orc.make_sw_loss(D.STRESS_WEIGHT, target), x, v)
    with _engine(x, v, box, prec, theta) as e:
        sig = e.stress()[0]
        e.set_loss(D.STRESS_WEIGHT, target)
        l, gx, gv, gp = e.loss_grad()
    assert nrel(sig, sig_ref) <= ftol
    assert abs(l[0] - l_ref) <= gtol * abs(l_ref)
    assert nrel(gx, gx_ref) <= gtol and nrel(gv, gv_ref) <= gtol
    assert group_err(gp[0], gp_ref) <= gtol, group_err(gp[0], gp_ref)


@pytest.mark.parametrize("prec,gtol", [("fp64", 1e-6), ("mixed", 1e-4)])
@pytest.mark.parametrize("trunc", [12, 3])
def test_reverse_gradient_matches_oracle(theta, prec, gtol, trunc):
    x, v, box = _crystal(3, 0.003)
    seeds = np.arange(1, 13, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    s = orc.make_sw_system(len(x), box, mlp=True)
    L = orc.make_sw_loss(D.STRESS_WEIGHT)
    xf, vf, lf, sx, sv = orc.sw_forward_sim(s, theta, x, v, seeds, 4.0, 12, 5, 0.0005, L)
    _, _, lr_ref, g_ref = orc.sw_reverse_sim(s, theta, xf, vf, seeds, 4.0, 12, 5, trunc, 0.0005, sx, sv, L)
    with _engine(x, v, box, prec, theta) as e:
        e.set_loss()
        lfw, nb = e.forward(seeds, 4.0, 12, 5, 0.0005)
        lrv, g = e.reverse(seeds, 4.0, 12, 5, trunc, 0.0005)
        xr, _ = e.get_state()
    assert nb == 3 and abs(lrv[0] - lfw[0]) <= 1e-12 * abs(lfw[0])
    assert abs(lrv[0] - lr_ref) <= gtol * abs(lr_ref)
    assert group_err(g[0], g_ref) <= gtol, group_err(g[0], g_ref)
    if trunc == 12:
        d = xr - x
        d -= np.round(d / box) * box
        assert np.abs(d).max() < (1e-8 if prec == "fp64" else 1e-6)


def test_zero_weights_are_the_plain_engine():
    x, v, box = _crystal()
    p = np.concatenate([D.default_params(), np.zeros(D.MLP_NPARAMS)])
    with _engine(x, v, box, "mixed", p) as e:
        F1 = e.forces()
    with SwEngine(len(x), box, precision="mixed") as e0:
        e0.set_params(D.default_params())
        e0.set_state(x, v)
        F0 = e0.forces()
    assert np.array_equal(F1, F0)   # u = 0 exactly: the same rounded sums


def test_batched_replicas_have_their_own_mlp_gradients(theta):
    systems = [_crystal(3, 0.003, seed=11), _crystal(4, 0.002, seed=12)]
    seeds = np.arange(1, 21, dtype=np.uint64).reshape(20, 1) * np.uint64(0x2545F4914F6CDD1D) + \
        np.arange(2, dtype=np.uint64).reshape(1, 2)
    singles = []
    for r, (x, v, box) in enumerate(systems):
        with _engine(x, v, box, "mixed", theta) as e:
            e.set_loss()
            e.forward(seeds[:, r], 1.0, 20, 10, 0.0005)
            singles.append(e.reverse(seeds[:, r], 1.0, 20, 10, 10, 0.0005)[1][0])
    eb = SwEngine([len(s[0]) for s in systems], [s[2] for s in systems], precision="mixed", mlp=True)
    eb.set_params(theta)
    eb.set_state(np.concatenate([s[0] for s in systems]), np.concatenate([s[1] for s in systems]))
    eb.set_loss()
    eb.forward(seeds, 1.0, 20, 10, 0.0005)
    _, g = eb.reverse(seeds, 1.0, 20, 10, 10, 0.0005)
    eb.close()
    for r in range(2):
        # the coefficient adjoints sum with FP64 atomics: equal to rounding
        assert group_err(g[r], singles[r]) <= 1e-10


def test_reference_entry_points_take_params_gnn(theta):
    from revsim import sw
    x, v, box = _crystal(3, 0.003)
    seeds = np.arange(1, 13, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
    sys_f, loss_f, acc, _, _, g_gnn0 = sw.forward_sim(x, v, seeds, 4.0, 12, 5, 0, theta[:7], theta[7:],
                                                       0.0005, box=box, precision="fp64")
    sys_r, loss_r, g_sw, g_gnn = sw.reverse_sim(sys_f.coords, sys_f.velocities, seeds, 4.0, 12, 5, 12, 0,
                                                theta[:7], theta[7:], 0.0005, 1, sys_f.loggers, acc)
    eng = sys_f.loggers
    assert eng.mlp and g_gnn0.shape == (D.MLP_NPARAMS,)
    assert abs(loss_r - loss_f) <= 1e-12 * abs(loss_f)
    assert g_sw.shape == (7,) and g_gnn.shape == (D.MLP_NPARAMS,) and np.abs(g_gnn).max() > 0
    with pytest.raises(ValueError):
        sw.forward_sim(x, v, seeds, 4.0, 12, 5, 0, theta[:7], None, 0.0005, engine=eng)
    eng.close()
