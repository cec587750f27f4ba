"""GPU parity: librevsim.so (through the C ABI) against the FP64 CPU oracle.

Tolerances (from the engine's contract):
* neighbour pair set: bit-exact;
* forces: 1e-10 relative (FP64 mode), 1e-5 relative (mixed), norm-wise;
* force VJP / dtheta contraction: 1e-10 (FP64), 1e-4 (mixed);
* reverse-pass gradients: 1e-6 (FP64) / 1e-4 (mixed) relative to the FP64 oracle,
  in units of dL/dlog(theta) floored at 1% of the largest component;
* reconstruction < 1e-9 nm and |L_rev - L_fwd| < 1e-7 in FP64 (water.jl:1613-1614).
"""

import numpy as np
import pytest

from conftest import relaxed_water
from oracle import orc
from revsim import Engine, RevsimError, constants as C, systems
from revsim.engine import RdfTerm
from revsim.loss import reference_rdf_terms

pytestmark = pytest.mark.gpu

FORMS = ["lj", "dexp", "buck", "ljsc", "buff"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    import build
    build.build()


def engine(n_mol, box, form="lj", prec="fp64", **kw):
    e = Engine(n_mol, box, inter_type=form, precision=prec, **kw)
    e.set_params(C.default_params(form))
    return e


def nrel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def min_image(d, box):
    return d - box * np.round(d / box)


def scaled_err(g, ref, p):
    s = np.abs(ref * p)
    return np.abs((g - ref) * p) / np.maximum(s, 0.01 * s.max())


def l2_terms(x, s, cut=0.04, n=200):
    t0 = orc.RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, cut, n, 0, 1, np.zeros(n), 2, 1.0)
    target = 0.9 * orc.rdf(s, t0, x) + 0.05
    otrm = orc.RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, cut, n, 0, 1, target, 2, 1.0)
    etrm = RdfTerm(0, 0, 1.0 / n, 1.0 / n, 0.0005, cut, n, 0, 1, target, 2, 1.0)
    return orc.Loss([otrm]), [etrm]


# ---------------------------------------------------------------- neighbour list
@pytest.mark.parametrize("fixture", ["small_water", "dense_water"])
def test_neighbor_pairs_bit_exact(request, fixture):
    n_mol, box, x, v = request.getfixturevalue(fixture)
    e = engine(n_mol, box)
    e.set_state(x, v)
    got = e.neighbor_pairs(0)
    ref = orc.neighbor_pairs(orc.make_system(n_mol, box), x)
    np.testing.assert_array_equal(got, ref)


def test_neighbor_pairs_replicas_and_small_cells():
    # three replicas, one with a box small enough that every cell is visited
    sizes, boxes = [60, 150, 400], [2.45, 2.6, 2.48]
    xs = [relaxed_water(m, b, seed=10 + i, steps=20)[0] for i, (m, b) in enumerate(zip(sizes, boxes))]
    e = Engine(sizes, boxes)
    e.set_params(C.default_params())
    e.set_state(np.concatenate(xs), np.zeros((3 * sum(sizes), 3)))
    for r in range(3):
        ref = orc.neighbor_pairs(orc.make_system(sizes[r], boxes[r]), xs[r])
        np.testing.assert_array_equal(e.neighbor_pairs(r), ref)


# ---------------------------------------------------------------------- forces
@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_forces(dense_water, form, prec, tol):
    n_mol, box, x, v = dense_water
    e = engine(n_mol, box, form, prec)
    e.set_state(x, v)
    F = e.forces()
    s = orc.make_system(n_mol, box, form)
    Fo = orc.forces(s, np.array(C.default_params(form)), x, orc.neighbor_pairs(s, x))
    assert nrel(F, Fo) < tol
    assert np.abs(F - Fo).max() < tol * np.abs(Fo).max()


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 1e-4)])
def test_force_vjp_and_param_contraction(dense_water, form, prec, tol):
    n_mol, box, x, v = dense_water
    rng = np.random.default_rng(7)
    w = rng.normal(size=x.shape)
    ac = rng.normal(size=x.shape)
    e = engine(n_mol, box, form, prec)
    e.set_state(x, v)
    F, G, th = e.force_vjp(w, ac)
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    Fo, Go, J = orc.forces_grads(s, p, x, orc.neighbor_pairs(s, x), w)
    tho = ac.ravel() @ J
    assert nrel(F, Fo) < (1e-10 if prec == "fp64" else 1e-5)
    assert nrel(G, Go) < tol
    assert np.all(scaled_err(th[0], tho, p) < tol), scaled_err(th[0], tho, p)


def test_forces_deterministic(dense_water):
    n_mol, box, x, v = dense_water
    for prec in ("fp64", "mixed"):
        e = engine(n_mol, box, "lj", prec)
        e.set_state(x, v)
        np.testing.assert_array_equal(e.forces(), e.forces())


def test_noise_matches_oracle():
    e = Engine([100, 50], [2.5, 2.5], temp=[280.0, 320.0])
    s0, s1 = orc.make_system(100, 2.5, temp=280.0), orc.make_system(50, 2.5, temp=320.0)
    xi = e.noise([12345, 999])
    np.testing.assert_allclose(xi[:300], orc.noise(s0, 12345), rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(xi[300:], orc.noise(s1, 999), rtol=1e-13, atol=1e-15)


# ------------------------------------------------------------------------ loss
def test_rdf_loss_and_gradient(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    ol, terms = l2_terms(x, s)
    e = engine(n_mol, box)
    e.set_state(x, v)
    e.set_loss(terms)
    h = e.rdf(0, 0)
    np.testing.assert_allclose(h, orc.rdf(s, ol.terms[0], x), rtol=1e-11, atol=1e-12)
    l, g = e.loss_grad()
    lo, go = orc.loss_grad(s, ol, x)
    assert abs(l[0] - lo) < 1e-10 * abs(lo)
    assert nrel(g, go) < 1e-10


def test_reference_rdf_loss_l1_oo_oh(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    rng = np.random.default_rng(1)
    t_oo, t_oh = rng.uniform(0, 2, 248), rng.uniform(0, 2, 281)
    terms = reference_rdf_terms(t_oo, t_oh)
    e = engine(n_mol, box)
    e.set_state(x, v)
    e.set_loss(terms)
    l, g = e.loss_grad()
    ol = orc.Loss([orc.RdfTerm(t.sel1, t.sel2, t.x_min, t.step, t.width, t.exp_cutoff, t.n_grid,
                               t.slice_start, t.slice_stride, t.target, t.norm, t.weight) for t in terms])
    lo, go = orc.loss_grad(s, ol, x)
    assert abs(l[0] - lo) < 1e-10 * abs(lo)
    assert nrel(g, go) < 1e-9


# ------------------------------------------------------------------ trajectories
def test_forward_trajectory_matches_oracle(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    seeds = systems.noise_seeds(10, seed=21)
    e = engine(n_mol, box)
    e.set_state(x, v)
    e.forward(seeds, 1.0, 10, 10, 0.001, calc_loss=False)
    xg, vg = e.get_state()
    xo, vo, _, _, _ = orc.forward_sim(s, p, x, v, seeds, 1.0, 10, 10, 0.001, None, False)
    assert np.abs(min_image(xg - xo, box)).max() < 1e-10
    assert np.abs(vg - vo).max() < 1e-8


@pytest.mark.parametrize("gamma", [1.0, 0.0])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_reverse_identities(dense_water, gamma, prec):
    n_mol, box, x, v = dense_water
    s = orc.make_system(n_mol, box)
    _, terms = l2_terms(x, s)
    e = engine(n_mol, box, "lj", prec)
    e.set_loss(terms)
    e.set_state(x, v)
    seeds = systems.noise_seeds(100, seed=31)
    lf = e.forward(seeds, gamma, 100, 100, 0.001)
    lr, g = e.reverse(seeds, gamma, 100, 100, 100, 0.001)
    xr, vr = e.get_state()
    recon = np.abs(min_image(xr - x, box)).max()
    assert recon < (1e-9 if prec == "fp64" else 1e-7), recon
    assert abs(lr[0] - lf[0]) < 1e-7
    assert np.all(np.isfinite(g))


@pytest.mark.parametrize("form", ["lj", "dexp", "buck"])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-6), ("mixed", 1e-4)])
def test_reverse_gradient_matches_oracle(small_water, form, prec, tol):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    ol, terms = l2_terms(x, s)
    n = 30
    seeds = systems.noise_seeds(n, seed=41)
    xf, vf, lfo, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, ol)
    _, _, lro, go = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, ol)
    e = engine(n_mol, box, form, prec)
    e.set_loss(terms)
    e.set_state(x, v)
    lf = e.forward(seeds, 1.0, n, n, 0.001)
    lr, g = e.reverse(seeds, 1.0, n, n, n, 0.001)
    assert abs(lf[0] - lfo) < (1e-10 if prec == "fp64" else 1e-5) * abs(lfo)
    err = scaled_err(g[0], go, p)
    # The exponential forms evaluate exp(alpha (1 - r/rm)) (alpha ~ 16.8) or exp(-B r)
    # (B = 27.6 nm^-1) in FP32, which amplifies the FP32 rounding of r: 3e-4 for those.
    if prec == "mixed" and form != "lj":
        tol = 3e-4
    assert np.all(err < tol), err


def test_blocks_truncation_and_snapshots(small_water):
    """Several loss blocks, truncated windows and snapshot restores (water.jl:1525-1547)."""
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    ol, terms = l2_terms(x, s)
    n, nl, tr, nlog = 60, 20, 10, 20
    seeds = systems.noise_seeds(n, seed=51)
    xf, vf, lfo, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, nl, 0.001, ol, n_steps_log=nlog)
    _, _, lro, go = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, tr, 0.001, sx, sv, ol, n_steps_log=nlog)
    e = engine(n_mol, box, n_steps_log=nlog)
    e.set_loss(terms)
    e.set_state(x, v)
    lf = e.forward(seeds, 1.0, n, nl, 0.001)
    lr, g = e.reverse(seeds, 1.0, n, nl, tr, 0.001)
    assert abs(lf[0] - lfo) < 1e-10 * abs(lfo)
    assert abs(lr[0] - lro) < 1e-9 * abs(lro)
    assert np.all(scaled_err(g[0], go, p) < 1e-6)


def test_neighbor_modes_and_clipping(small_water):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    ol, terms = l2_terms(x, s)
    n = 40
    seeds = systems.noise_seeds(n, seed=61)
    out = {}
    for mode in ("checkpoint", "reconstructed"):
        e = engine(n_mol, box, nl_mode=mode)
        e.set_loss(terms)
        e.set_state(x, v)
        e.forward(seeds, 1.0, n, n, 0.001)
        out[mode] = e.reverse(seeds, 1.0, n, n, n, 0.001)[1][0]
    assert np.all(scaled_err(out["checkpoint"], out["reconstructed"], p) < 1e-9)
    # clipping of dl_dfi by its norm (water.jl:1511-1515) against the oracle
    xf, vf, _, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, ol)
    clip = 1e-3
    _, _, _, go = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, ol, clip=clip)
    e = engine(n_mol, box)
    e.set_loss(terms)
    e.set_state(x, v)
    e.forward(seeds, 1.0, n, n, 0.001)
    g = e.reverse(seeds, 1.0, n, n, n, 0.001, clip=clip)[1][0]
    assert np.all(scaled_err(g, go, p) < 1e-6)


def test_batched_replicas_equal_single_runs():
    sizes, boxes, temps = [150, 90, 200], [2.6, 2.5, 2.7], [280.0, 300.0, 320.0]
    xs, vs = zip(*[relaxed_water(m, b, seed=70 + i, steps=30) for i, (m, b) in enumerate(zip(sizes, boxes))])
    n = 20
    seeds = np.stack([systems.noise_seeds(n, seed=80 + r) for r in range(3)], axis=1)
    terms_all = []
    for r in range(3):
        _, t = l2_terms(xs[r], orc.make_system(sizes[r], boxes[r]))
        terms_all.append(t[0].target)
    eb = Engine(sizes, boxes, temp=temps)
    eb.set_params(C.default_params())
    eb.set_loss([RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, np.stack(terms_all), 2, 1.0)])
    eb.set_state(np.concatenate(xs), np.concatenate(vs))
    lfb = eb.forward(seeds, 1.0, n, n, 0.001)
    lrb, gb = eb.reverse(seeds, 1.0, n, n, n, 0.001)
    for r in range(3):
        e = Engine(sizes[r], boxes[r], temp=temps[r])
        e.set_params(C.default_params())
        e.set_loss([RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, terms_all[r], 2, 1.0)])
        e.set_state(xs[r], vs[r])
        lf = e.forward(seeds[:, r], 1.0, n, n, 0.001)
        lr, g = e.reverse(seeds[:, r], 1.0, n, n, n, 0.001)
        # The RDF histogram sums with FP64 atomics, so losses agree to rounding only.
        assert abs(lf[0] - lfb[r]) < 1e-13 * abs(lf[0]) and abs(lr[0] - lrb[r]) < 1e-13 * abs(lr[0])
        assert np.all(scaled_err(gb[r], g[0], np.array(C.default_params())) < 1e-10)


# ----------------------------------------------------------------- failure paths
def test_device_checks_report_errors(small_water):
    n_mol, box, x, v = small_water
    e = engine(n_mol, box)
    bad = x.copy()
    bad[1] = bad[0] + np.array([0.2, 0.0, 0.0])   # an O-H bond of 0.2 nm
    e.set_state(bad, v)
    with pytest.raises(RevsimError) as ei:
        e.forces()
    assert ei.value.code == -6
    nan = x.copy()
    nan[4, 0] = np.nan
    e.set_state(nan, v)
    with pytest.raises(RevsimError) as ei:
        e.forces()
    assert ei.value.code in (-4, -6)
    e.set_state(x, v)
    e.forces()   # the handle stays usable


def test_argument_errors(small_water):
    n_mol, box, x, v = small_water
    e = engine(n_mol, box)
    e.set_state(x, v)
    seeds = systems.noise_seeds(10)
    with pytest.raises(RevsimError) as ei:
        e.reverse(seeds, 1.0, 10, 10, 10, 0.001)
    assert ei.value.code == -7   # no loss set / no forward pass
    _, terms = l2_terms(x, orc.make_system(n_mol, box))
    e.set_loss(terms)
    with pytest.raises(RevsimError) as ei:
        e.reverse(seeds, 1.0, 10, 5, 6, 0.001)
    assert ei.value.code == -1
    with pytest.raises(RevsimError):
        e.set_params([1.0, 2.0])
    with pytest.raises(RevsimError):
        Engine(10, 2.0)   # box below twice the neighbour cutoff


# ------------------------------------------- 3.0 nm box: one image per molecule pair
@pytest.mark.parametrize("form", ["lj", "buck"])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_forces_and_vjp_box3(cfg1_water, form, prec, tol):
    n_mol, box, x, v = cfg1_water
    rng = np.random.default_rng(8)
    w, ac = rng.normal(size=x.shape), rng.normal(size=x.shape)
    e = engine(n_mol, box, form, prec)
    e.set_state(x, v)
    F = e.forces()
    F2, G, th = e.force_vjp(w, ac)
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    Fo, Go, J = orc.forces_grads(s, p, x, orc.neighbor_pairs(s, x), w)
    assert nrel(F, Fo) < tol and nrel(F2, Fo) < tol
    assert nrel(G, Go) < 10 * tol
    assert np.all(scaled_err(th[0], ac.ravel() @ J, p) < 10 * tol)


def test_launch_shapes_agree(cfg1_water):
    n_mol, box, x, v = cfg1_water
    rng = np.random.default_rng(9)
    w, ac = rng.normal(size=x.shape), rng.normal(size=x.shape)
    e = engine(n_mol, box, "lj", "fp64")
    e.set_state(x, v)
    ref = None
    per_g = {}
    for G in (8, 16, 32):
        shapes = [(threads // G, U) for threads in (64, 256, 512) for U in (1, 2, 3)
                  if not (U == 3 and threads > 256)]
        for mpc, U in shapes:
            e.set_launch_shape(G, mpc, U)
            F, Gv, th = e.force_vjp(w, ac)
            if ref is None:
                ref = (F, Gv, th)
            assert nrel(F, ref[0]) < 1e-13 and nrel(Gv, ref[1]) < 1e-13
            assert np.all(scaled_err(th[0], ref[2][0], np.array(C.default_params())) < 1e-12)
            # at one lane count every loop form sums each atom's slots in the same order
            if G in per_g:
                assert np.array_equal(F, per_g[G][0]) and np.array_equal(Gv, per_g[G][1]), (G, mpc, U)
            else:
                per_g[G] = (F, Gv)
    rshape, fshape = e.autotune()
    assert rshape[0] in (8, 16, 32) and rshape[2] in (1, 2, 3) and fshape[0] in (8, 16, 32)
    F2, Gv2, _ = e.force_vjp(w, ac)
    assert nrel(F2, ref[0]) < 1e-13 and nrel(Gv2, ref[1]) < 1e-13


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-6), ("mixed", 1e-4)])
def test_reverse_gradient_box3(cfg1_water, prec, tol):
    """This box is hot (~720 K after a short relaxation from the lattice): within one
    20-step list lifetime some pairs come within 1.0 nm without having been within
    1.2 nm at the list build, so the reference's schedule (forward lists built from
    x_{20k}, reverse lists rebuilt from reconstructed x_{20k-1}, water.jl:1038,1504)
    interacts different pair sets in the two passes.  The engine's reconstructed-list
    mode follows that schedule and is compared with the oracle here; its default
    checkpoint mode reuses the forward lists (compared on equilibrated boxes above)."""
    n_mol, box, x, v = cfg1_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    ol, terms = l2_terms(x, s)
    n = 20
    seeds = systems.noise_seeds(n, seed=91)
    xf, vf, lfo, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, ol)
    _, _, _, go = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, ol)
    e = engine(n_mol, box, "lj", prec, nl_mode="reconstructed")
    e.set_loss(terms)
    e.set_state(x, v)
    e.forward(seeds, 1.0, n, n, 0.001)
    lr, g = e.reverse(seeds, 1.0, n, n, n, 0.001)
    assert np.all(scaled_err(g[0], go, p) < tol), scaled_err(g[0], go, p)
    # Different pair sets forward and backward also cost the reconstruction its
    # 1e-9 accuracy on this box (for the reference as much as for the engine).
    xr, _ = e.get_state()
    assert np.abs(min_image(xr - x, box)).max() < 1e-3


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_forces_with_molecules_across_faces(cfg1_water, prec, tol):
    """Atoms are wrapped one by one, so molecules straddle the box faces; shifting the
    box origin puts hundreds of them across a face at once."""
    n_mol, box, x, v = cfg1_water
    xs = x + 1.47
    xs -= np.floor(xs / box) * box
    raw = xs[1::3] - xs[0::3]
    assert (np.abs(raw) > box / 2).any(axis=1).sum() > 10
    e = engine(n_mol, box, "lj", prec)
    e.set_state(xs, v)
    F = e.forces()
    s = orc.make_system(n_mol, box)
    Fo = orc.forces(s, np.array(C.default_params()), xs, orc.neighbor_pairs(s, xs))
    assert nrel(F, Fo) < tol
    np.testing.assert_array_equal(e.neighbor_pairs(0), orc.neighbor_pairs(s, xs))
