"""The enthalpy-of-vaporisation loss term on the GPU (revsim_set_enth_vap, loss_type :enth_vap
and :both of loss_fn, water.jl:738-769) against the FP64 oracle (orc_loss_and_grads,
orc_forward_sim / orc_reverse_sim with the term on).

Bars: the loss and its parts 1e-10 relative (the energy kernel is FP64 in both precision
modes); dL/dx 1e-10 (FP64) / 1e-5 (mixed: the (2 e / n) F term uses the mode's forces);
the direct dl/dtheta 1e-10 (1e-9 with the learned term); reverse-pass gradients 1e-6 (FP64) /
1e-4 (mixed) in units of dL/dlog(theta) floored at 1% of the largest component, as the
RDF-loss parity tests; batched replicas equal to single runs to 1e-10; the reweighting
estimator with the enthalpy term against the oracle's over the same run to 1e-6.
"""

import numpy as np
import pytest

from conftest import relaxed_water
from oracle import orc
from revsim import Engine, constants as C, mlp, systems
from revsim.water import forward_sim, reverse_sim, reweighting_sim

from test_gpu_parity import l2_terms, nrel, scaled_err

pytestmark = pytest.mark.gpu

FORMS = ["lj", "dexp", "buck", "ljsc", "buff"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def _losses(s, x, rdf):
    ol, terms = l2_terms(x, s)
    return orc.Loss(ol.terms if rdf else [], enth_vap=True), (terms if rdf else [])


def _engine(n_mol, box, form, prec, terms, p=None, **kw):
    e = Engine(n_mol, box, inter_type=form, precision=prec, **kw)
    e.set_params(C.default_params(form) if p is None else p)
    e.set_loss(terms)
    e.set_enth_vap(True)
    return e


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("form", FORMS)
def test_loss_and_grads_match_oracle(dense_water, form, prec):
    n_mol, box, x, v = dense_water
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    ol, terms = _losses(s, x, rdf=True)
    lo, (lro, leo), go, dpo = orc.loss_and_grads(s, p, ol, x)
    e = _engine(n_mol, box, form, prec, terms)
    e.set_state(x, v)
    l, lr, le, g, dp = e.loss_and_grads()
    l2, g2 = e.loss_grad()
    e.close()
    assert leo > 0 and lro > 0
    assert abs(l[0] - lo) <= 1e-10 * lo and abs(le[0] - leo) <= 1e-10 * leo
    assert abs(lr[0] - lro) <= 1e-10 * lo
    assert nrel(g, go) <= (1e-10 if prec == "fp64" else 1e-5)
    # the RDF histogram and its gradient sum with FP64 atomics: equal to rounding
    assert abs(l2[0] - l[0]) <= 1e-13 * l[0] and nrel(g2, g) <= 1e-13
    assert np.abs(dp[0] - dpo).max() <= 1e-10 * np.abs(dpo).max()


def test_direct_gradient_with_the_learned_term(dense_water):
    n_mol, box, x, v = dense_water
    th = mlp.init_params(3) + np.random.default_rng(4).normal(scale=0.05, size=mlp.N_PARAMS)
    p = np.concatenate([C.default_params("lj"), th])
    s = orc.make_system(n_mol, box, "lj", mlp=True)
    ol = orc.Loss([], enth_vap=True)
    lo, _, go, dpo = orc.loss_and_grads(s, p, ol, x)
    e = _engine(n_mol, box, "lj", "fp64", [], p=p, mlp=True)
    e.set_state(x, v)
    l, lr, le, g, dp = e.loss_and_grads()
    e.close()
    assert abs(l[0] - lo) <= 1e-9 * lo and lr[0] == 0.0
    assert nrel(g, go) <= 1e-10
    assert np.abs(dp[0, :7] - dpo[:7]).max() <= 1e-9 * np.abs(dpo[:7]).max()
    assert np.abs(dp[0, 7:] - dpo[7:]).max() <= 1e-9 * np.abs(dpo[7:]).max()


@pytest.mark.parametrize("rdf", [False, True])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-6), ("mixed", 1e-4)])
def test_reverse_gradient_matches_oracle(small_water, rdf, prec, tol):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    ol, terms = _losses(s, x, rdf)
    n, nl = 40, 20
    seeds = systems.noise_seeds(n, seed=41)
    xf, vf, lfo, sx, sv, (fro, feo) = orc.forward_sim(s, p, x, v, seeds, 1.0, n, nl, 0.001, ol,
                                                      n_steps_log=20, parts=True)
    _, _, lro, go = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, nl, 0.001, sx, sv, ol,
                                    n_steps_log=20)
    e = _engine(n_mol, box, "lj", prec, terms, n_steps_log=20)
    e.set_state(x, v)
    lf = e.forward(seeds, 1.0, n, nl, 0.001)
    fr, fe = e.loss_parts()
    lr, g = e.reverse(seeds, 1.0, n, nl, nl, 0.001)
    rr, re = e.loss_parts()
    e.close()
    ftol = 1e-10 if prec == "fp64" else 1e-5
    assert abs(lf[0] - lfo) <= ftol * lfo and abs(fe[0] - feo) <= ftol * feo
    assert abs(fr[0] - fro) <= ftol * lfo
    assert abs(lr[0] - lf[0]) <= 1e-7 * lf[0] and abs(re[0] - fe[0]) <= 1e-7 * fe[0]
    err = scaled_err(g[0], go, p)
    assert np.all(err < tol), err


def test_reference_signature_loss_types(small_water):
    """forward_sim / reverse_sim with loss_type "rdf", "enth_vap" and "both" on one engine:
    the parts add up, and the :both loss is the sum of the two single-term losses."""
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    _, terms = l2_terms(x, s)
    p = np.array(C.default_params())
    n = 20
    seeds = systems.noise_seeds(n, seed=9)
    out = {}
    eng = None
    for lt in ("rdf", "enth_vap", "both"):
        sys_f, lf, _ = forward_sim(x, v, box, seeds, 1.0, n, n, p, 0.001, 1, "lj", lt,
                                   loss_terms=terms if eng is None else None, engine=eng)
        eng = sys_f.engine
        sys_r, lr, g, l_rdf, l_ev = reverse_sim(sys_f.coords, sys_f.velocities, box, seeds, 1.0, n, n,
                                                n, p, 0.001, 1, sys_f.loggers, None, "lj", lt)
        assert abs(lr - lf) <= 1e-9 * lf and abs(l_rdf + l_ev - lr) <= 1e-12 * lr
        out[lt] = (lr, g, l_rdf, l_ev)
    eng.close()
    assert out["rdf"][3] == 0.0 and out["enth_vap"][2] == 0.0
    assert abs(out["both"][0] - out["rdf"][0] - out["enth_vap"][0]) <= 1e-10 * out["both"][0]
    # the gradient of a sum of losses is the sum of the gradients
    assert np.all(scaled_err(out["both"][1], out["rdf"][1] + out["enth_vap"][1], p) < 1e-8)
    with pytest.raises(ValueError):
        forward_sim(x, v, box, seeds, 1.0, n, n, p, 0.001, 1, "lj", "density")


def test_batched_replicas_equal_single_runs():
    sizes, boxes, temps = [150, 90], [2.6, 2.5], [280.0, 310.0]
    xs, vs = zip(*[relaxed_water(m, b, seed=70 + i, steps=30) for i, (m, b) in enumerate(zip(sizes, boxes))])
    n = 20
    seeds = np.stack([systems.noise_seeds(n, seed=80 + r) for r in range(2)], axis=1)
    eb = _engine(sizes, boxes, "lj", "fp64", [], temp=temps)
    eb.set_state(np.concatenate(xs), np.concatenate(vs))
    lfb = eb.forward(seeds, 1.0, n, 10, 0.001)
    lrb, gb = eb.reverse(seeds, 1.0, n, 10, 10, 0.001)
    eb.close()
    p = np.array(C.default_params())
    for r in range(2):
        e = _engine(sizes[r], boxes[r], "lj", "fp64", [], temp=temps[r])
        e.set_state(xs[r], vs[r])
        lf = e.forward(seeds[:, r], 1.0, n, 10, 0.001)
        lr, g = e.reverse(seeds[:, r], 1.0, n, 10, 10, 0.001)
        e.close()
        assert abs(lf[0] - lfb[r]) <= 1e-12 * lf[0] and abs(lr[0] - lrb[r]) <= 1e-12 * lr[0]
        assert np.all(scaled_err(gb[r], g[0], p) < 1e-10)


def test_reweighting_estimator_with_the_enthalpy_term(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box, "lj")
    p = np.array(C.default_params("lj"))
    ol, terms = _losses(s, x, rdf=True)
    n_steps, nl = 60, 20
    seeds = systems.noise_seeds(n_steps, seed=17)
    # the oracle estimator over the same run (water.jl:1159-1207)
    xo, vo = x.copy(), v.copy()
    L, Le, dl, dE, LdE = 0.0, 0.0, np.zeros(7), np.zeros(7), np.zeros(7)
    for b in range(n_steps // nl):
        xo, vo, _, _, _ = orc.forward_sim(s, p, xo, vo, seeds[b * nl:(b + 1) * nl], 1.0, nl, nl,
                                          0.001, ol)
        lb, (_, leb), _, dlb = orc.loss_and_grads(s, p, ol, xo)
        _, gb = orc.energy_grads(s, p, xo, orc.neighbor_pairs(s, xo))
        L += lb
        Le += leb
        dl += dlb
        dE += gb
        LdE += lb * gb
    nb = n_steps // nl
    beta = 1.0 / (C.KB * C.TEMP)
    g_ref = dl / nb - beta * (LdE / nb - (L / nb) * dE / nb)
    sys, loss, grads, l_rdf, l_ev = reweighting_sim(x, v, box, seeds, 1.0, n_steps, nl, p, 0.001, 1,
                                                    "lj", "both", loss_terms=terms, precision="fp64")
    sys.engine.close()
    assert abs(loss - L / nb) <= 1e-8 * (L / nb) and abs(l_ev - Le / nb) <= 1e-8 * (Le / nb)
    assert abs(l_rdf + l_ev - loss) <= 1e-12 * loss
    assert np.abs(grads - g_ref).max() <= 1e-6 * np.abs(g_ref).max(), (grads, g_ref)
