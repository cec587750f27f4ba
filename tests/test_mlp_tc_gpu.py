"""The learned term's network on the tensor cores (revsim_set_mlp_precision REVSIM_MLP_BF16_TC:
BF16 operands, each FP32 value split into a BF16 high part and a BF16 remainder and every
product formed by three MMAs with FP32 accumulation) against the FP64 oracle and the FP64
kernels.  Split operands carry ~16 significant bits, so the bars are:
* node values u and du/dr of all three types: max error <= 1e-3 of the largest |u|, |du/dr|;
* at arbitrary distances (a per-pair evaluation): the same bar against the oracle's table
  interpolant, which is < 1e-8 from the exact network;
* the weight gradient from the same interval-coefficient adjoints (a force VJP at the same
  positions: the adjoints do not depend on the table values): per layer group (W1 + b1,
  W2 + b2, w3 + b3 of each type) the relative L2 error against the FP64 backward <= 1e-2 and
  the cosine >= 0.9999 (the gradients are node sums whose terms largely cancel);
* the reverse-pass gradient of a 20-step run, which also sees the two tables' different
  dynamics: classical parameters within 5e-3 of the FP64-network run (parameter-scaled as the
  classical tests), MLP groups within 1e-2 / 0.9999.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import Engine, RdfTerm, RevsimError, constants as C, mlp, systems

from test_mlp_gpu import groups

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


@pytest.fixture(scope="module")
def theta():
    th = mlp.init_params(3)
    th += np.random.default_rng(4).normal(scale=0.05, size=th.shape)
    return np.concatenate([C.default_params("lj"), th])


def _engine(n_mol, box, theta, mode, prec="fp64"):
    e = Engine(n_mol, box, precision=prec, mlp=True)
    e.set_mlp_precision(mode)
    e.set_params(theta)
    return e


def _groups_close(a_all, b_all):
    for ix in groups(len(b_all))[1:]:
        a, b = a_all[ix], b_all[ix]
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b), (ix[0], np.linalg.norm(a - b) / np.linalg.norm(b))
        assert a @ b >= 0.9999 * np.linalg.norm(a) * np.linalg.norm(b)


def test_tc_nodes_match_oracle(small_water, theta):
    n_mol, box, x, v = small_water
    e = _engine(n_mol, box, theta, "bf16_tc")
    u, du = e.mlp_eval()
    uo, duo = orc.mlp_nodes(theta[7:])
    assert np.abs(u - uo).max() <= 1e-3 * np.abs(uo).max(), np.abs(u - uo).max() / np.abs(uo).max()
    assert np.abs(du - duo).max() <= 1e-3 * np.abs(duo).max()


def test_tc_per_pair_evaluation(small_water, theta):
    n_mol, box, x, v = small_water
    e = _engine(n_mol, box, theta, "bf16_tc")
    r = np.random.default_rng(5).uniform(0.05, 1.0, size=(3, 777))
    u, du = e.mlp_eval(r)
    coef = orc.mlp_table(theta[7:])
    uo = np.array([[orc.mlp_pair(coef, t, rr)[0] for rr in r[t]] for t in range(3)])
    Fo = np.array([[orc.mlp_pair(coef, t, rr)[1] for rr in r[t]] for t in range(3)])
    assert np.abs(u - uo).max() <= 1e-3 * np.abs(uo).max()
    assert np.abs(-du - Fo).max() <= 1e-3 * np.abs(Fo).max()


def test_tc_backward_matches_fp64(small_water, theta):
    n_mol, box, x, v = small_water
    rng = np.random.default_rng(6)
    w, ac = rng.normal(size=x.shape), rng.normal(size=x.shape)
    out = {}
    for mode in ("fp64", "bf16_tc"):
        e = _engine(n_mol, box, theta, mode)
        e.set_state(x, v)
        out[mode] = e.force_vjp(w, ac)[2][0]
        e.close()
    _groups_close(out["bf16_tc"], out["fp64"])


def test_tc_reverse_gradient(small_water, theta):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    n = 20
    seeds = systems.noise_seeds(n, seed=8)
    out = {}
    for mode in ("fp64", "bf16_tc"):
        e = _engine(n_mol, box, theta, mode, prec="mixed")
        e.set_loss([RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
        e.set_state(x, v)
        e.forward(seeds, 1.0, n, n, 0.001)
        out[mode] = e.reverse(seeds, 1.0, n, n, n, 0.001)[1][0]
        e.close()
    g64, gtc = out["fp64"], out["bf16_tc"]
    p = theta[:7]
    sc = np.abs(g64[:7] * p)
    assert np.all(np.abs((gtc[:7] - g64[:7]) * p) / np.maximum(sc, 0.01 * sc.max()) < 5e-3)
    _groups_close(gtc, g64)


def test_mlp_precision_argument_checks(small_water, theta):
    n_mol, box, x, v = small_water
    e = Engine(n_mol, box)
    e.set_params(C.default_params())
    with pytest.raises(RevsimError):
        e.set_mlp_precision("bf16_tc")      # no learned term on this handle
    e2 = _engine(n_mol, box, theta, "fp64")
    with pytest.raises(RevsimError):
        e2._check(e2._L.revsim_set_mlp_precision(e2.handle, 7))
