"""Host-side logic: generators, loss builders, parameter layout, data parsing."""

import numpy as np

from revsim import constants as C, loss, systems


def test_lattice_and_geometry():
    assert systems.lattice_dims(895) == (10, 10, 9)
    x = systems.water_coords(895, 3.0, seed=0)
    assert x.shape == (2685, 3) and np.all(x >= 0) and np.all(x < 3.0)
    o, h1, h2 = x[0::3], x[1::3], x[2::3]

    def mi(d):
        return d - 3.0 * np.round(d / 3.0)
    a, b = mi(h1 - o), mi(h2 - o)
    np.testing.assert_allclose(np.linalg.norm(a, axis=1), C.R0_BOND, rtol=1e-12)
    cos = (a * b).sum(1) / (np.linalg.norm(a, axis=1) * np.linalg.norm(b, axis=1))
    np.testing.assert_allclose(np.arccos(cos), C.THETA0_ANGLE, rtol=1e-10)
    np.testing.assert_array_equal(x, systems.water_coords(895, 3.0, seed=0))


def test_velocities_and_seeds():
    v = systems.mb_velocities(3000, temp=295.15, seed=1)
    m = systems.masses(3000)
    T = (m[:, None] * v * v).sum() / (3 * 9000 * C.KB)
    assert abs(T - 295.15) / 295.15 < 0.03
    s = systems.noise_seeds(10, seed=2)
    assert s.dtype == np.uint64 and len(set(s.tolist())) == 10


def test_param_layout():
    assert C.default_params("lj") == [0.315, 0.636, -0.834, 462750.4, 0.09572, 836.8, 1.82421813418]
    for t in C.INTER_TYPES:
        assert len(C.default_params(t)) == C.n_params(t)


def test_reference_rdf_terms_slices():
    terms = loss.reference_rdf_terms(np.zeros(248), np.zeros(281))
    oo, oh = terms
    # water.jl:708-709: 323:6:1805 and 125:6:1805 (1-based) on 0.1:0.0005:2.5
    assert oo.slice_start + 6 * 247 == 1804 and oh.slice_start + 6 * 280 == 1804
    assert abs(oo.x_min + oo.step * 322 - 0.261) < 1e-12
    assert abs(oh.x_min + oh.step * 124 - 0.162) < 1e-12
    assert oo.n_grid == 4801


def test_read_rdf_data(tmp_path):
    p = tmp_path / "rdf.txt"
    rows = ["0.00 0 0 0 0 0 0", "0.01 0 0 0 0 0 0"]
    rows += [f"{0.02 + 0.003 * i:.3f} {i} 0 {i + 1000} 0 {i + 2000} 0" for i in range(400)]
    p.write_text("\n".join(rows) + "\n")
    oo, oh, hh = loss.read_rdf_data(str(p))
    assert len(oo) == 248 and len(oh) == 281 and len(hh) == 261
    assert oo[0] == 86 and oh[0] == 1053 and hh[0] == 2073


def test_l2_term_grid():
    t = loss.oo_l2_term(np.zeros(200))
    assert t.x_min == t.step == 0.005 and t.n_grid == 200 and t.norm == 2
