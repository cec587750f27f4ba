"""Chained step launches change no result: the same forward + reverse run, in a process
with REVSIM_CHAIN=0 (plain stream serialisation) and in one with chaining on, gives
bit-identical trajectories — water (mixed and FP64, Langevin noise, neighbour rebuilds, two
loss blocks), Stillinger-Weber diamond (mixed and FP64, stress loss, four blocks) and gas in
water (FP64, diffusion + enthalpy loss, where losses and gradients are bit-identical too).
The water and diamond losses and gradients are compared with tolerances.  The water RDF loss and its dL/dx are FP64 atomic sums whose order
varies from run to run, so the water losses are compared to 1e-12 relative and the
gradients to 1e-10 (FP64) and 1e-5 (mixed: an FP64 adjoint that differs in its last bit may
round to a different FP32 operand).

Each run is a child process because the switch is read once per process."""

import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import PKG, ROOT, relaxed_gas, relaxed_water

pytestmark = pytest.mark.gpu

CHILD = r"""
import sys
import numpy as np
from revsim import Engine, constants as C, systems
from revsim.engine import RdfTerm
from revsim.gas import GasEngine

d = np.load(sys.argv[1])
out = {}
n_mol, box = int(d["n_mol"]), float(d["box"])
n = 200
target = np.full(200, 1.0)
terms = [RdfTerm(0, 0, 1.0 / 200, 1.0 / 200, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)]
for prec in ("mixed", "fp64"):
    e = Engine(n_mol, box, precision=prec)
    e.set_params(C.default_params())
    e.set_loss(terms)
    e.set_state(d["wx"], d["wv"])
    seeds = systems.noise_seeds(n, seed=5)
    lf = e.forward(seeds, 1.0, n, 100, 0.001)
    out[prec + "_xf"], out[prec + "_vf"] = e.get_state()
    lr, g = e.reverse(seeds, 1.0, n, 100, 100, 0.001)
    x, v = e.get_state()
    out[prec + "_lf"] = np.asarray(lf, dtype=np.float64)
    out[prec + "_lr"] = np.asarray(lr, dtype=np.float64)
    out[prec + "_g"] = np.asarray(g, dtype=np.float64)
    out[prec + "_x"] = x
    out[prec + "_v"] = v
from revsim import SwEngine, diamond as D
sx, sbox = D.diamond_coords(3, noise=0.003, seed=4)
sv = D.mb_velocities(len(sx), seed=5)
sseeds = np.arange(1, 41, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
for prec in ("mixed", "fp64"):
    with SwEngine(len(sx), sbox, precision=prec) as se:
        se.set_params(D.default_params())
        se.set_state(sx, sv)
        se.set_loss()
        lf, _ = se.forward(sseeds, 4.0, 40, 10, 0.0005)
        out["sw" + prec + "_xf"], out["sw" + prec + "_vf"] = se.get_state()
        lr, g = se.reverse(sseeds, 4.0, 40, 10, 10, 0.0005)
        out["sw" + prec + "_x"], out["sw" + prec + "_v"] = se.get_state()
        out["sw" + prec + "_lf"] = np.asarray(lf, dtype=np.float64)
        out["sw" + prec + "_lr"] = np.asarray(lr, dtype=np.float64)
        out["sw" + prec + "_g"] = np.asarray(g, dtype=np.float64)
ge = GasEngine(int(d["n_water"]), int(d["n_gas"]), float(d["gbox"]))
ge.set_params(d["gp"])
ge.set_state(d["gx"], d["gv"])
seeds = systems.noise_seeds(n, seed=9)
lf, parts_f, centres = ge.forward(seeds, 1.0, n, 50, 0.001, "diff_ev")
out["gas_xf"], out["gas_vf"] = ge.get_state()
lr, g, parts_r = ge.reverse(seeds, 1.0, n, 50, 20, 0.001, "diff_ev")
x, v = ge.get_state()
out.update(gas_lf=np.array([lf]), gas_pf=parts_f, gas_c=centres, gas_lr=np.array([lr]),
           gas_g=g, gas_pr=parts_r, gas_x=x, gas_v=v)
np.savez(sys.argv[2], **out)
"""


def _run(tmp_path, inp, chain):
    outp = str(tmp_path / f"out_{chain}.npz")
    env = dict(os.environ)
    env["REVSIM_CHAIN"] = chain
    env["PYTHONPATH"] = os.pathsep.join([PKG, ROOT, env.get("PYTHONPATH", "")])
    r = subprocess.run([sys.executable, "-c", CHILD, inp, outp], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(outp)


def test_chained_launches_bit_identical(tmp_path):
    import build
    build.build()
    wx, wv = relaxed_water(150, 2.6, seed=0, steps=100)
    s, gp, gx, gv = relaxed_gas(80, 5, 2.5, seed=4, steps=30)
    inp = str(tmp_path / "in.npz")
    np.savez(inp, n_mol=150, box=2.6, wx=wx, wv=wv, n_water=s.n_water, n_gas=s.n_gas, gbox=s.box,
             gp=gp, gx=gx, gv=gv)
    plain = _run(tmp_path, inp, "0")
    chained = _run(tmp_path, inp, "1")
    assert sorted(plain.files) == sorted(chained.files)
    for k in plain.files:
        assert np.all(np.isfinite(plain[k])), k
        prec, what = k.split("_")
        if prec != "gas" and what in ("lf", "lr", "g"):
            tol = 1e-12 if what != "g" else (1e-10 if prec.endswith("fp64") else 1e-5)
            scale = np.abs(plain[k]).max()
            assert np.abs(chained[k] - plain[k]).max() <= tol * scale, k
        else:
            assert plain[k].tobytes() == chained[k].tobytes(), k
