"""Constants and seeded generators of the Stillinger-Weber diamond system (host side, numpy).

Values follow greener-group/rev-sim ``diamond/diamond.jl``:

* carbon mass 12.011 u, temperature 298 K, 1,000 atoms in a 1.784 nm box (5^3 cells):
  ``diamond.jl:38-52``
* SW parameters theta = [A, B, a, lambda, gamma, sigma, eps] and exponents p = 4, q = 0:
  ``diamond.jl:53`` and ``diamond.jl:1352-1356``
* stress-loss weight gamma_sigma = 5e-8 (kJ/mol)^-2 nm^6: ``diamond.jl:57``

The reference builds its start lattice with SimpleCrystals.Diamond (``diamond.jl:1397-1399``);
here the same conventional 8-atom cell is tiled and jittered from a seed.
"""

import numpy as np

C_MASS = 12.011
TEMP = 298.0
KB = 0.00831446261815324
SIDE_LENGTH = 1.784
LATTICE_A = 0.3567
STRESS_WEIGHT = 5e-8
PARAM_NAMES = ("A", "B", "a", "lambda", "gamma", "sigma", "eps")
N_PARAMS = 7
# The learned radial term (one MLP type of revsim.mlp on [0, 0.25 nm], RBF width 0.0125 nm):
# its parameters follow the SW ones when the engine has it.
MLP_CUTOFF, MLP_WIDTH = 0.25, 0.0125
MLP_NPARAMS = 5313


def init_mlp_params(seed=3):
    """Seeded initialisation of the learned radial term (the first type of
    revsim.mlp.init_params)."""
    from . import mlp
    return mlp.init_params(seed)[:MLP_NPARAMS]


def default_params():
    """Initial SW parameters of diamond.jl:53."""
    return np.array([7.049556277, 0.6022245584, 1.80, 21.0, 1.20, 0.14, 200.0])


# Fractional coordinates of the conventional diamond cell (FCC + (1/4, 1/4, 1/4) basis).
_CELL = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0],
                  [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75],
                  [0.75, 0.75, 0.25]])


def diamond_coords(n_cells, a=LATTICE_A, noise=0.0, seed=4):
    """Positions [8 n_cells^3, 3] (nm) of an n_cells^3 diamond lattice in a cubic box of side
    n_cells * a, with seeded Gaussian displacement of standard deviation ``noise`` per axis,
    wrapped into [0, box).  Returns (x, box)."""
    n = int(n_cells)
    ii, jj, kk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    origins = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1).astype(np.float64)
    x = ((origins[:, None, :] + _CELL[None, :, :]) * a).reshape(-1, 3)
    box = n * a
    if noise > 0:
        x = x + np.random.default_rng(seed).normal(scale=noise, size=x.shape)
    return x - np.floor(x / box) * box, box


def mb_velocities(n_atoms, temp=TEMP, seed=5, mass=C_MASS):
    """Maxwell-Boltzmann velocities [n_atoms, 3] (nm/ps) with the mean removed."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n_atoms, 3)) * np.sqrt(KB * temp / mass)
    return v - v.mean(axis=0)
