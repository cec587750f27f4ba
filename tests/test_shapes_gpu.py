"""Launch shapes and reversibility.

The order in which a molecule's pair forces are summed depends on the lanes per molecule
(a lane takes every G-th entry of the row; a G-lane butterfly sums the lanes), so the
forward and the reverse step kernels give the same force bits only at the same lane count.
The reverse pass rebuilds the forward trajectory only from the same force bits (in mixed
precision a one-ulp FP32 difference is amplified by the dynamics), so the lane count is one
setting for both kernels and the autotuner chooses it jointly.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import Engine, RdfTerm, RevsimError, constants as C, systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def _engine(n_mol, box, prec):
    e = Engine(n_mol, box, precision=prec)
    e.set_params(C.default_params())
    return e


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_autotuned_kernels_give_the_same_force_bits(dense_water, prec):
    n_mol, box, x, v = dense_water
    e = _engine(n_mol, box, prec)
    e.set_state(x, v)
    rshape, fshape = e.autotune()
    assert rshape[0] == fshape[0]
    rng = np.random.default_rng(2)
    F_fwd = e.forces()                                     # forward-kernel shape
    F_rev, _, _ = e.force_vjp(rng.normal(size=x.shape), rng.normal(size=x.shape))   # reverse
    np.testing.assert_array_equal(F_fwd, F_rev)


def test_lane_count_is_shared(dense_water):
    n_mol, box, x, v = dense_water
    e = _engine(n_mol, box, "mixed")
    e.set_launch_shape(32, 16, 1, which=1)                 # forward: 512 threads
    e.set_launch_shape(16, 8, 3, which=0)                  # reverse: 128 threads, U = 3
    assert e.launch_shape(0) == (16, 8, 3)
    assert e.launch_shape(1) == (16, 16, 1)                # the forward kernel follows
    e.set_launch_shape(8, 64, 1, which=1)                  # both at 8 lanes: 512 / 64 threads
    assert e.launch_shape(0) == (8, 8, 3)
    with pytest.raises(RevsimError):
        e.set_launch_shape(16, 0, 0, which=0)              # forward would need 1,024 threads
    assert e.launch_shape(1) == (8, 64, 1) and e.launch_shape(0) == (8, 8, 3)


def test_mixed_reconstruction_with_autotuned_shapes(dense_water):
    n_mol, box, x, v = dense_water
    s = orc.make_system(n_mol, box)
    t0 = orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.zeros(200), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    e = _engine(n_mol, box, "mixed")
    e.set_loss([RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, target, 2, 1.0)])
    e.set_state(x, v)
    e.autotune()
    # 100 steps, the reference's own self-check length (water.jl:1613): over longer untruncated
    # windows the FP64 rounding of the reconstruction grows with the dynamics' chaos until it
    # moves some position across an FP32 rounding boundary, after which the two passes' forces
    # differ by an ulp
    n = 100
    seeds = systems.noise_seeds(n, seed=14)
    e.set_state(x, v)
    e.forward(seeds, 0.0, n, n, 0.001)
    e.reverse(seeds, 0.0, n, n, n, 0.001)
    x0, v0 = e.get_state()
    d = x0 - x
    d -= box * np.round(d / box)
    assert np.abs(d).max() < 1e-7, np.abs(d).max()
    assert np.abs(v0 - v).max() < 1e-5
