"""Committed fixtures (tests/golden/water_small.npz, made by tests/golden/make_golden.py).

CPU: the oracle still reproduces them (OpenMP reduction order may move the last bits,
hence 1e-12).  GPU: the engine, through the C ABI, against the same fixed numbers, with
the parity tolerances of tests/test_gpu_parity.py.
"""

import os

import numpy as np
import pytest

from oracle import orc
from revsim import constants as C

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "water_small.npz")
FORMS = ["lj", "dexp", "buck", "ljsc", "buff"]


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def test_oracle_reproduces_fixtures(gold):
    n, box, x = int(gold["n_mol"]), float(gold["box"]), gold["x"]
    s = orc.make_system(n, box)
    pairs = orc.neighbor_pairs(s, x)
    np.testing.assert_array_equal(pairs, gold["pairs"])
    for f in FORMS:
        sf = orc.make_system(n, box, f)
        pf = np.array(C.default_params(f))
        F, G, J = orc.forces_grads(sf, pf, x, pairs, gold["w"])
        assert rel(orc.forces(sf, pf, x, pairs), gold[f"forces_{f}"]) < 1e-12
        assert rel(G, gold[f"vjp_{f}"]) < 1e-12
        assert rel(gold["acoef"].ravel() @ J, gold[f"dtheta_{f}"]) < 1e-12
    np.testing.assert_array_equal(orc.noise(s, int(gold["noise_seed"])), gold["noise"])
    t = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, gold["target"], 2, 1.0)
    assert rel(orc.rdf(s, t, x), gold["rdf"]) < 1e-12
    l, g = orc.loss_grad(s, orc.Loss([t]), x)
    assert abs(l - gold["loss"]) < 1e-12 * abs(gold["loss"]) and rel(g, gold["dLdx"]) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_engine_matches_fixtures(gold, prec, tol):
    import build
    build.build()
    from revsim import Engine, RdfTerm
    n, box, x, v = int(gold["n_mol"]), float(gold["box"]), gold["x"], gold["v"]
    for f in FORMS:
        e = Engine(n, box, inter_type=f, precision=prec)
        e.set_params(C.default_params(f))
        e.set_state(x, v)
        if f == "lj":
            np.testing.assert_array_equal(e.neighbor_pairs(0), gold["pairs"])
        assert rel(e.forces(), gold[f"forces_{f}"]) < tol
        _, G, th = e.force_vjp(gold["w"], gold["acoef"])
        assert rel(G, gold[f"vjp_{f}"]) < 10 * tol
        assert rel(th[0], gold[f"dtheta_{f}"]) < 10 * tol
        e.close()
    e = Engine(n, box, precision=prec)
    e.set_params(C.default_params())
    e.set_state(x, v)
    np.testing.assert_allclose(e.noise(int(gold["noise_seed"])), gold["noise"], rtol=1e-13, atol=1e-15)
    e.set_loss([RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, gold["target"], 2, 1.0)])
    np.testing.assert_allclose(e.rdf(0, 0), gold["rdf"], rtol=1e-11, atol=1e-12)
    seeds = gold["seeds"]
    nst = len(seeds)
    lf = e.forward(seeds, 1.0, nst, nst, 0.001)
    assert abs(lf[0] - gold["fwd_loss"]) < (1e-9 if prec == "fp64" else 1e-4) * abs(gold["fwd_loss"])
    lr, g = e.reverse(seeds, 1.0, nst, nst, nst, 0.001)
    p = np.array(C.default_params())
    sc = np.abs(gold["rev_grad"] * p)
    err = np.abs((g[0] - gold["rev_grad"]) * p) / np.maximum(sc, 0.01 * sc.max())
    assert np.all(err < (1e-6 if prec == "fp64" else 1e-4)), err
