"""Seeded water-box generators and a TIP3P PDB loader (host side, numpy).

The reference starts from ``water/tip3p.pdb`` (895 HOH in a 3.0 nm box,
``water.jl:33-34``).  Benchmarks and tests use seeded synthetic boxes of the same
chemistry: molecules on a jittered lattice with uniformly random orientations and
Maxwell-Boltzmann velocities.  Atom order is O, H1, H2 per molecule, as in the PDB.
"""

import math

import numpy as np

from . import constants as C


def lattice_dims(n_mol):
    """Smallest n x n x m lattice holding n_mol sites (895 -> 10 x 10 x 9)."""
    n = max(1, math.ceil(round(n_mol ** (1.0 / 3.0), 9)))
    while n**3 < n_mol:
        n += 1
    m = math.ceil(n_mol / (n * n))
    return n, n, m


def _random_rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def water_coords(n_mol, box, seed=0, jitter=0.02, r0=C.R0_BOND, theta0=C.THETA0_ANGLE):
    """Positions [3*n_mol, 3] (nm) wrapped into [0, box)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = lattice_dims(n_mol)
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    sites = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)[:n_mol].astype(np.float64)
    sites = (sites + 0.5) * (box / np.array([nx, ny, nz], dtype=np.float64))
    sites += rng.uniform(-jitter, jitter, size=sites.shape)
    h = 0.5 * theta0
    local = np.array([[0.0, 0.0, 0.0],
                      [r0 * math.sin(h), 0.0, r0 * math.cos(h)],
                      [-r0 * math.sin(h), 0.0, r0 * math.cos(h)]])
    R = _random_rotations(rng, n_mol)
    x = sites[:, None, :] + np.einsum("mab,kb->mka", R, local)
    x = x.reshape(-1, 3)
    return x - np.floor(x / box) * box


def masses(n_mol):
    return np.tile(np.array([C.O_MASS, C.H_MASS, C.H_MASS]), n_mol)


def mb_velocities(n_mol, temp=C.TEMP, seed=1):
    """Maxwell-Boltzmann velocities [3*n_mol, 3] (nm/ps)."""
    rng = np.random.default_rng(seed)
    sd = np.sqrt(C.KB * temp / masses(n_mol))
    return rng.normal(size=(3 * n_mol, 3)) * sd[:, None]


def noise_seeds(n_steps, seed=0):
    """Per-step 64-bit noise seeds (the reference draws rand(0:typemax(Int)),
    water.jl:875; here they are seeded for reproducibility)."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, np.iinfo(np.int64).max, size=n_steps, dtype=np.int64).astype(np.uint64)


def load_pdb(path):
    """Coordinates [N, 3] in nm and the cubic box side from a CRYST1/ATOM PDB."""
    box = None
    xs = []
    with open(path) as f:
        for line in f:
            if line.startswith("CRYST1"):
                box = float(line[6:15]) / 10.0
            elif line.startswith(("ATOM", "HETATM")):
                xs.append([float(line[30:38]), float(line[38:46]), float(line[46:54])])
    x = np.asarray(xs, dtype=np.float64) / 10.0
    if box is not None:
        x = x - np.floor(x / box) * box
    return x, box


def box_for_density(n_mol, mol_per_nm3=33.1):
    """Cubic box side giving liquid-water number density (~33.1 molecules/nm^3)."""
    return (n_mol / mol_per_nm3) ** (1.0 / 3.0)


def gas_water_coords(n_water, n_gas, box, seed=0, jitter=0.02):
    """Waters followed by O2 molecules [3 n_water + 2 n_gas, 3] (nm), wrapped.  As in
    setup_system (diffusion.jl:1060-1118): n_water + n_gas lattice waters, n_gas of them
    (chosen by the seed) become O2 with the first site on the water O and the second
    0.12074 nm along O -> H1."""
    n_mol = n_water + n_gas
    x = water_coords(n_mol, box, seed=seed, jitter=jitter).reshape(n_mol, 3, 3)
    rng = np.random.default_rng(seed + 1000)
    gas = np.sort(rng.choice(n_mol, size=n_gas, replace=False))
    keep = np.setdiff1d(np.arange(n_mol), gas)
    xo = x[gas, 0]
    d = x[gas, 1] - xo
    d -= box * np.round(d / box)
    o2 = xo + d / np.linalg.norm(d, axis=1, keepdims=True) * C.GAS_R0_BOND
    out = np.concatenate([x[keep].reshape(-1, 3), np.stack([xo, o2], axis=1).reshape(-1, 3)])
    return out - np.floor(out / box) * box


def gas_water_masses(n_water, n_gas):
    return np.concatenate([masses(n_water), np.full(2 * n_gas, C.O_MASS)])


def gas_water_velocities(n_water, n_gas, temp=C.TEMP, seed=1):
    """Maxwell-Boltzmann velocities of the gas-in-water system (nm/ps)."""
    rng = np.random.default_rng(seed)
    sd = np.sqrt(C.KB * temp / gas_water_masses(n_water, n_gas))
    return rng.normal(size=(len(sd), 3)) * sd[:, None]
