"""Generate tests/golden/water_small.npz from the FP64 CPU oracle.

The reference (Julia) cannot run on these machines and ships no golden vectors, so these
fixtures are outputs of the oracle (oracle/revsim_oracle.c), itself pinned by the
reference's identities and central differences (tests/test_oracle.py).  They freeze the
oracle's results for a small seeded system so that regressions in the oracle and GPU
parity can be checked against fixed numbers.

    python tests/golden/make_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "rev-sim_b200"))

from oracle import orc  # noqa: E402
from revsim import constants as C, systems  # noqa: E402

N_MOL, BOX = 100, 2.5
FORMS = ["lj", "dexp", "buck", "ljsc", "buff"]


def make():
    x = systems.water_coords(N_MOL, BOX, seed=21)
    v = systems.mb_velocities(N_MOL, seed=22)
    s = orc.make_system(N_MOL, BOX)
    p = np.array(C.default_params())
    x, v, _, _, _ = orc.forward_sim(s, p, x, v, systems.noise_seeds(40, seed=23), 1.0, 40, 40, 0.001,
                                    None, False)
    out = {"x": x, "v": v, "n_mol": N_MOL, "box": BOX}
    pairs = orc.neighbor_pairs(s, x)
    out["pairs"] = pairs
    rng = np.random.default_rng(24)
    w = rng.normal(size=x.shape)
    ac = rng.normal(size=x.shape)
    out["w"], out["acoef"] = w, ac
    for f in FORMS:
        sf = orc.make_system(N_MOL, BOX, f)
        pf = np.array(C.default_params(f))
        F, G, J = orc.forces_grads(sf, pf, x, pairs, w)
        out[f"forces_{f}"] = orc.forces(sf, pf, x, pairs)
        out[f"vjp_{f}"] = G
        out[f"dtheta_{f}"] = ac.ravel() @ J
    out["noise_seed"] = np.uint64(12345)
    out["noise"] = orc.noise(s, 12345)
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    h = orc.rdf(s, t0, x)
    out["rdf"] = h
    target = 0.9 * h + 0.05
    out["target"] = target
    loss = orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
    l, g = orc.loss_grad(s, loss, x)
    out["loss"], out["dLdx"] = l, g
    n = 30
    seeds = systems.noise_seeds(n, seed=25)
    out["seeds"] = seeds
    xf, vf, lf, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, loss)
    out["fwd_x"], out["fwd_v"], out["fwd_loss"] = xf, vf, lf
    xr, vr, lr, gr = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, loss)
    out["rev_x"], out["rev_loss"], out["rev_grad"] = xr, lr, gr
    return out


if __name__ == "__main__":
    orc.build()
    d = make()
    np.savez_compressed(os.path.join(HERE, "water_small.npz"), **d)
    print("wrote", os.path.join(HERE, "water_small.npz"))
