"""Shared test setup: import paths, the gpu marker, and small seeded systems."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rev-sim_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


def pytest_collection_modifyitems(config, items):
    # Keep file order (a test file named test_zz_* runs last).
    items.sort(key=lambda it: (os.path.basename(str(it.fspath)),))


def relaxed_water(n_mol, box, seed=0, steps=100, inter_type="lj"):
    """A seeded lattice box relaxed by the oracle with Langevin steps (gamma = 1/ps)."""
    from oracle import orc
    from revsim import constants as C, systems

    x = systems.water_coords(n_mol, box, seed=seed)
    v = systems.mb_velocities(n_mol, seed=seed + 1)
    s = orc.make_system(n_mol, box, inter_type)
    p = np.array(C.default_params(inter_type))
    if steps:
        x, v, _, _, _ = orc.forward_sim(s, p, x, v, systems.noise_seeds(steps, seed=seed + 7), 1.0,
                                        steps, steps, 0.001, None, False)
    return x, v


def relaxed_gas(n_water, n_gas, box, inter_type="lj", seed=0, steps=60):
    """A seeded gas-in-water box relaxed by the oracle with Langevin steps (gamma = 1/ps):
    (oracle system, default parameters, x, v)."""
    from oracle import orc
    from revsim import constants as C, systems

    s = orc.make_gas_system(n_water, n_gas, box, inter_type)
    x = systems.gas_water_coords(n_water, n_gas, box, seed=seed)
    v = systems.gas_water_velocities(n_water, n_gas, seed=seed + 1)
    p = np.array(C.gas_default_params(inter_type))
    if steps:
        x, v, *_ = orc.gas_forward_sim(s, p, x, v, systems.noise_seeds(steps, seed=seed + 7), 1.0,
                                       steps, steps, 0.001, calc_loss=False)
    return s, p, x, v


@pytest.fixture(scope="session")
def small_water():
    """150 molecules in a 2.6 nm box (low density keeps the oracle fast), relaxed."""
    x, v = relaxed_water(150, 2.6, seed=0, steps=100)
    return 150, 2.6, x, v


@pytest.fixture(scope="session")
def dense_water():
    """400 molecules in a 2.48 nm box (liquid density), relaxed."""
    x, v = relaxed_water(400, 2.48, seed=3, steps=100)
    return 400, 2.48, x, v


@pytest.fixture(scope="session")
def cfg1_water():
    """895 molecules in a 3.0 nm box (the reference's tip3p.pdb size), relaxed."""
    x, v = relaxed_water(895, 3.0, seed=5, steps=60)
    return 895, 3.0, x, v
