"""Generate tests/golden/reference_inputs.npz from the reference's own input files.

The reference runs its water gradient on `water/tip3p.pdb` (895 HOH in a 3.0 nm box,
water.jl:32) and ships the parameter sets it trained in `water/trained_force_fields/*.xml`.
The GPU box has no copy of the reference, so this script reads those files here and
stores what the tests need: the 2,685 positions as `revsim.systems.load_pdb` reads them
(nm, O H1 H2 per molecule, wrapped into the box as wrap_coords does at water.jl:1037),
the box side from CRYST1, and per parameter set the flat parameter vector in the layout of
water.jl:1572-1582 (pair form, then q_O, k_b, r0, k_a, theta0):

* tip3p      -- Molly's tip3p_standard.xml that water.jl:28-32 loads (the repo's copy,
                trained_force_fields/tip3p.xml), as the LJ form;
* lj, lj_reweighting -- NonbondedForce sigma/epsilon of the O type (LJ form);
* buckingham -- CustomNonbondedForce A, B, C of the O type;
* double_exponential -- sigma, epsilon of the O type and the global alpha, beta;
* lj_soft_core -- sigma, epsilon of the O type and the global alpha, lambda.

    python tests/golden/make_reference_inputs.py [reference water directory]
"""

import os
import sys
import xml.etree.ElementTree as ET

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rev-sim_b200"))
OUT = os.path.join(HERE, "reference_inputs.npz")
DEFAULT_SRC = "/root/reference/water"

# file -> (pair form of the engine, pair-form parameter names)
SETS = {
    "tip3p": ("tip3p.xml", "lj"),
    "lj": ("lj.xml", "lj"),
    "lj_reweighting": ("lj_reweighting.xml", "lj"),
    "buckingham": ("buckingham.xml", "buck"),
    "double_exponential": ("double_exponential.xml", "dexp"),
    "lj_soft_core": ("lj_soft_core.xml", "ljsc"),
}


def _o_atom(section):
    for a in section.findall("Atom"):
        if a.get("type") == "tip3p-O":
            return a
    raise ValueError("no tip3p-O entry")


def read_params(path, form):
    root = ET.parse(path).getroot()
    charge = None
    for res in root.iter("Residue"):
        if res.get("name") == "HOH":
            charge = float(next(a for a in res.findall("Atom") if a.get("name") == "O").get("charge"))
    bond = next(b for b in root.iter("Bond") if b.get("type1") == "tip3p-O" and b.get("type2") == "tip3p-H")
    angle = next(a for a in root.iter("Angle") if a.get("type2") == "tip3p-O")
    tail = [charge, float(bond.get("k")), float(bond.get("length")), float(angle.get("k")),
            float(angle.get("angle"))]
    if form == "lj":
        o = _o_atom(root.find("NonbondedForce"))
        head = [float(o.get("sigma")), float(o.get("epsilon"))]
    else:
        cnb = root.find("CustomNonbondedForce")
        o = _o_atom(cnb)
        glob = {g.get("name"): float(g.get("defaultValue")) for g in cnb.findall("GlobalParameter")}
        if form == "buck":
            head = [float(o.get("A")), float(o.get("B")), float(o.get("C"))]
        elif form == "dexp":
            head = [float(o.get("sigma")), float(o.get("epsilon")), glob["α"], glob["β"]]
        else:   # ljsc
            head = [float(o.get("sigma")), float(o.get("epsilon")), glob["α"], glob["λ"]]
    return np.array(head + tail)


def make(src=DEFAULT_SRC):
    from revsim import systems
    x, box = systems.load_pdb(os.path.join(src, "tip3p.pdb"))
    out = {"x_tip3p": x, "box_tip3p": np.float64(box)}
    for name, (fname, form) in SETS.items():
        out[f"params_{name}"] = read_params(os.path.join(src, "trained_force_fields", fname), form)
        out[f"form_{name}"] = np.array(form)
    return out


if __name__ == "__main__":
    d = make(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC)
    np.savez(OUT, **d)
    print(OUT, {k: v.shape for k, v in d.items()})
