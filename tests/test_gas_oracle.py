"""The gas-in-water oracle (diffusion.jl restated): its derivatives by central differences,
F = -dU/dx, the diffusion coefficient's gradient, and the reverse pass against the forward
loss (the reference's own checks, diffusion.jl:1659-1677)."""

import numpy as np
import pytest

from conftest import relaxed_gas
from oracle import orc
from revsim import systems

FORMS = ["lj", "dexp", "buck", "ljsc", "buff"]


@pytest.fixture(scope="module")
def small_gas():
    return relaxed_gas(120, 6, 2.6)


def test_pairs_exclude_molecules_and_match_brute_force(small_gas):
    s, p, x, v = small_gas
    pairs = orc.gas_neighbor_pairs(s, x)
    n = orc.gas_n_atoms(s)
    mol = np.concatenate([np.repeat(np.arange(s.n_water), 3),
                          s.n_water + np.repeat(np.arange(s.n_gas), 2)])
    d = x[None, :, :] - x[:, None, :]
    d -= s.box * np.round(d / s.box)
    r2 = (d * d).sum(-1)
    i, j = np.triu_indices(n, 1)
    keep = (r2[i, j] <= 1.2 ** 2) & (mol[i] != mol[j])
    ref = np.stack([i[keep], j[keep]], axis=1)
    assert np.array_equal(pairs, ref)


@pytest.mark.parametrize("form", FORMS)
def test_forces_are_minus_energy_gradient(form):
    s, p, x, _ = relaxed_gas(60, 4, 2.5, form, seed=2, steps=20)
    pairs = orc.gas_neighbor_pairs(s, x)
    F = orc.gas_forces(s, p, x, pairs)
    rng = np.random.default_rng(1)
    for a in rng.choice(orc.gas_n_atoms(s), size=6, replace=False):
        for u in range(3):
            h = 1e-6
            xp, xm = x.copy(), x.copy()
            xp[a, u] += h
            xm[a, u] -= h
            fd = -(orc.gas_energy(s, p, xp, pairs) - orc.gas_energy(s, p, xm, pairs)) / (2 * h)
            assert abs(fd - F[a, u]) <= 2e-5 * max(1.0, abs(F[a, u])), (form, a, u)


@pytest.mark.parametrize("form", FORMS)
def test_vjp_and_contraction_by_central_differences(form):
    s, p, x, _ = relaxed_gas(60, 4, 2.5, form, seed=3, steps=20)
    pairs = orc.gas_neighbor_pairs(s, x)
    n = orc.gas_n_atoms(s)
    rng = np.random.default_rng(4)
    w = rng.normal(size=(n, 3))
    ac = rng.normal(size=(n, 3))
    F, G, dp = orc.gas_forces_grads(s, p, x, w, ac, pairs)
    assert np.allclose(F, orc.gas_forces(s, p, x, pairs), rtol=1e-12, atol=1e-9)
    m = systems.gas_water_masses(s.n_water, s.n_gas)[:, None]
    # u . G = (w/m) . dF/dx u
    for _ in range(3):
        u = rng.normal(size=(n, 3))
        h = 1e-7
        dF = (orc.gas_forces(s, p, x + h * u, pairs) - orc.gas_forces(s, p, x - h * u, pairs)) / (2 * h)
        lhs, rhs = (u * G).sum(), ((w / m) * dF).sum()
        assert abs(lhs - rhs) <= 1e-5 * max(abs(rhs), 1.0), (form, lhs, rhs)
    # dl_dp[k] = acoef . dF/dtheta_k
    for k in range(len(p)):
        h = 1e-5 * max(abs(p[k]), 1e-3)
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (ac * (orc.gas_forces(s, pp, x, pairs) - orc.gas_forces(s, pm, x, pairs))).sum() / (2 * h)
        assert abs(fd - dp[k]) <= 2e-5 * max(abs(fd), 1e-3 * np.abs(dp).max()), (form, k, fd, dp[k])


@pytest.mark.parametrize("form", FORMS)
def test_energy_parameter_gradient(form):
    s, p, x, _ = relaxed_gas(60, 4, 2.5, form, seed=5, steps=10)
    pairs = orc.gas_neighbor_pairs(s, x)
    E, dE = orc.gas_energy(s, p, x, pairs, grads=True)
    for k in range(len(p)):
        h = 1e-4 * abs(p[k])
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (orc.gas_energy(s, pp, x, pairs) - orc.gas_energy(s, pm, x, pairs)) / (2 * h)
        assert abs(fd - dE[k]) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(dE).max()), (form, k)


def test_mixing_rules_follow_the_sites():
    """A gas site with the water parameters makes the system the water model's pair set."""
    s, p, x, _ = relaxed_gas(60, 4, 2.5, "lj", seed=6, steps=5)
    pw = p.copy()
    pw[2], pw[3] = pw[0], pw[1]
    pairs = orc.gas_neighbor_pairs(s, x)
    E = orc.gas_energy(s, pw, x, pairs)
    # the same energy by hand: LJ between every non-H site pair within the cutoff
    nw3 = 3 * s.n_water
    sites = [a for a in range(orc.gas_n_atoms(s)) if a >= nw3 or a % 3 == 0]
    d = x[sites][None] - x[sites][:, None]
    d -= s.box * np.round(d / s.box)
    r = np.sqrt((d * d).sum(-1))
    pair_set = {(int(i), int(j)) for i, j in pairs}
    e_lj = 0.0
    for a_i, a in enumerate(sites):
        for b_i in range(a_i + 1, len(sites)):
            b = sites[b_i]
            if (a, b) in pair_set and r[a_i, b_i] <= 1.0:
                sr6 = (pw[0] / r[a_i, b_i]) ** 6
                e_lj += 4 * pw[1] * (sr6 * sr6 - sr6)
    pz = pw.copy()
    pz[1] = pz[3] = 0.0
    assert abs((E - orc.gas_energy(s, pz, x, pairs)) - e_lj) <= 1e-9 * abs(e_lj)


def test_diffusion_coefficient_and_its_gradient():
    rng = np.random.default_rng(7)
    box, lf = 2.6, 0.5
    gc = np.cumsum(rng.normal(scale=0.05, size=(7, 5, 3)), axis=0) + rng.uniform(0, box, (1, 5, 3))
    gc -= box * np.floor(gc / box)
    D, g = orc.gas_diffusion_D(gc, box, lf, grads=True)
    # unwrapped displacement over n_frames // 2 frames from every start frame
    ns = 3
    ref = 0.0
    for st in range(ns):
        d = gc[st + ns] - gc[st]
        d -= box * np.round(d / box)
        tot = np.zeros_like(d)
        for j in range(st + 1, st + ns + 1):
            dj = gc[j] - gc[j - 1]
            tot += dj - box * np.round(dj / box)
        ref += (tot ** 2).sum(-1).mean() / (ns * lf)
    assert abs(D - ref / (6 * ns)) <= 1e-12 * abs(D)
    assert np.all(g[6] == 0) and np.abs(g[:3]).max() > 0   # frame 6 is never an end frame here
    for f, q, u in [(0, 1, 2), (3, 4, 0), (5, 2, 1), (4, 0, 0)]:
        h = 1e-7
        gp, gm = gc.copy(), gc.copy()
        gp[f, q, u] += h
        gm[f, q, u] -= h
        fd = (orc.gas_diffusion_D(gp, box, lf) - orc.gas_diffusion_D(gm, box, lf)) / (2 * h)
        assert abs(fd - g[f, q, u]) <= 1e-6 * max(abs(fd), 1e-8)


@pytest.mark.parametrize("loss_type", ["diff", "diff_ev", "diff_rdf_ev"])
def test_reverse_reconstructs_and_matches_forward(small_gas, loss_type):
    """diffusion.jl:1674-1675: reconstruction < 1e-9, |L_rev - L_fwd| < 1e-7."""
    s, p, x0, v0 = small_gas
    n, nl = 40, 10
    seeds = systems.noise_seeds(n, seed=11)
    rdf = gas_rdf_loss(2) if "rdf" in loss_type else None
    xf, vf, lf, sx, sv, gc, outf = orc.gas_forward_sim(s, p, x0, v0, seeds, 1.0, n, nl, 0.001, loss_type,
                                                       rdf=rdf)
    xr, vr, lr, dp, outr = orc.gas_reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, nl, 0.001, sx, sv, gc,
                                               loss_type, rdf=rdf)
    d = xr - x0
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < 1e-9
    assert abs(lr - lf) < 1e-7 and np.isfinite(dp).all()
    assert np.allclose(outr, outf, rtol=1e-12, atol=0)


def gas_rdf_loss(seed=0):
    """Two smooth (squared-error) RDF terms over the water atoms, O-O and O-H, against seeded
    random targets: the shape of loss_rdf (diffusion.jl:759-774) without the Soper data."""
    rng = np.random.default_rng(seed)
    return orc.Loss([orc.RdfTerm(0, 0, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, rng.uniform(0, 2, 200), 2, 1.0),
                     orc.RdfTerm(0, 1, 0.005, 0.005, 0.0005, 0.04, 200, 0, 1, rng.uniform(0, 2, 200), 2, 1.0)])


def blockwise_fd(s, p, sx, sv, seeds, nl, n_blocks, loss_type, dl_dgc, k, rdf=None):
    """d/dtheta_k of the reverse pass's estimator by central differences: reverse_sim resets
    its adjoints at every loss point (diffusion.jl:1589-1605), so each loss point's gradient
    flows back through its own block only; here each block restarts from its stored snapshot
    with theta +- h and the frame's centres (and RDF / enthalpy terms) are differenced.  h is
    1e-3 relative: the centres move by ~1e-8 nm per 1e-5 of a parameter, where rounding
    dominates."""
    h = 1e-3 * abs(p[k])
    point = "_".join(t for t in ("rdf", "ev") if t in loss_type) or "ev"
    tot = 0.0
    for b in range(n_blocks):
        res = []
        for sgn in (1, -1):
            pk = p.copy()
            pk[k] += sgn * h
            out = orc.gas_forward_sim(s, pk, sx[b], sv[b], seeds[b * nl:(b + 1) * nl], 1.0, nl, nl,
                                      0.001, point, calc_loss=point in loss_type, rdf=rdf)
            res.append((out[5][0], (out[6][2] + out[6][3]) / n_blocks))
        d = res[0][0] - res[1][0]
        d -= s.box * np.round(d / s.box)
        tot += (dl_dgc[b] * d).sum() / (2 * h)
        if point in loss_type:
            tot += (res[0][1] - res[1][1]) / (2 * h)
    return tot


@pytest.mark.parametrize("form,loss_type", [("lj", "diff"), ("lj", "diff_ev"), ("buck", "diff"),
                                            ("dexp", "diff"), ("lj", "diff_rdf_ev"), ("lj", "rdf")])
def test_reverse_gradient_against_blockwise_central_differences(form, loss_type):
    """The reverse pass's gradient against central differences of the same estimator (the
    reference prints its reverse gradient beside RAD and FD ones, diffusion.jl:1656-1681)."""
    s, p, x0, v0 = relaxed_gas(60, 4, 2.5, form, seed=8, steps=30)
    n, nl = 24, 6
    rdf = gas_rdf_loss(3) if "rdf" in loss_type else None
    seeds = systems.noise_seeds(n, seed=13)
    xf, vf, lf, sx, sv, gc, _ = orc.gas_forward_sim(s, p, x0, v0, seeds, 1.0, n, nl, 0.001, loss_type,
                                                    rdf=rdf)
    _, _, lr, dp, _ = orc.gas_reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, nl, 0.001, sx, sv, gc,
                                          loss_type, rdf=rdf)
    assert abs(lr - lf) < 1e-7
    _, _, dl_dgc = orc.gas_loss_final("diff", gc, s.box, nl * 0.001)
    if "diff" not in loss_type:
        dl_dgc = np.zeros_like(dl_dgc)
    fd = np.array([blockwise_fd(s, p, sx, sv, seeds, nl, n // nl, loss_type, dl_dgc, k, rdf)
                   for k in range(len(p))])
    # in units of dL/dlog(theta), floored at 1% of the largest component
    sf = np.abs(fd * p)
    err = np.abs((dp - fd) * p) / np.maximum(sf, 0.01 * sf.max())
    assert np.all(err < 1e-4), (form, err)


def test_rdf_term_is_the_water_rdf_of_the_water_atoms():
    """The gas system's RDF loss point is the water restatement's loss on the water atoms,
    weighted 0.05 / n_blocks (diffusion.jl:51, 765-771)."""
    s, p, x0, v0 = relaxed_gas(60, 4, 2.5, seed=9, steps=10)
    rdf = gas_rdf_loss(4)
    n, nl = 12, 6
    seeds = systems.noise_seeds(n, seed=14)
    _, _, lf, sx, sv, gc, out = orc.gas_forward_sim(s, p, x0, v0, seeds, 1.0, n, nl, 0.001, "rdf", rdf=rdf)
    ws = orc.make_system(s.n_water, s.box)
    ref = sum(orc.loss_grad(ws, rdf, sx[b + 1].reshape(-1, 3)[:3 * s.n_water])[0] for b in range(2))
    assert abs(out[2] - 0.05 * ref / 2) <= 1e-12 * abs(out[2]) and out[1] == out[3] == 0.0
    assert abs(lf - out[2]) <= 1e-15 * abs(lf)
