"""The oracle's enthalpy-of-vaporisation loss (loss_enth_vap, water.jl:738-755, through
loss_fn / loss_and_grads, water.jl:757-786) against its definition and central differences:
the loss value from the potential energy, dL/dx and the direct dl/dtheta, and the reverse
gradient of a run with the enthalpy term (alone and with the RDF term) against central
differences of the forward loss.
"""

import numpy as np
import pytest

from oracle import orc
from revsim import constants as C, systems

from test_oracle import _fd_loss_grad, _scaled_err, _smooth_loss


def _ev_loss(s, x, rdf=True):
    """The RDF term of the oracle tests plus the enthalpy term (loss_type :both), or the
    enthalpy term alone (:enth_vap)."""
    terms = _smooth_loss(s, x, 0.14).terms if rdf else []
    return orc.Loss(terms, enth_vap=True)


def test_enthalpy_loss_value(small_water):
    n_mol, box, x, _ = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    U = orc.energy(s, p, x, orc.neighbor_pairs(s, x))
    dh = 3.69 - U / n_mol + 2.45          # enthalpy_vaporization, water.jl:738-746
    l, (l_rdf, l_ev), _, _ = orc.loss_and_grads(s, p, _ev_loss(s, x, rdf=False), x)
    assert l_rdf == 0.0
    assert abs(l_ev - (dh - 46.92) ** 2) <= 1e-12 * l_ev
    assert l == l_ev
    l2, (l_rdf2, l_ev2), _, _ = orc.loss_and_grads(s, p, _ev_loss(s, x), x)
    l_only, _ = orc.loss_grad(s, _smooth_loss(s, x, 0.14), x, False)
    assert l_rdf2 == l_only and l_ev2 == l_ev and l2 == l_rdf2 + l_ev2


@pytest.mark.parametrize("rdf", [False, True])
def test_enthalpy_loss_position_gradient(small_water, rdf):
    n_mol, box, x, _ = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    loss = _ev_loss(s, x, rdf)
    _, _, g, _ = orc.loss_and_grads(s, p, loss, x)
    u = np.random.default_rng(3).normal(size=x.shape)
    h = 1e-7
    fd = (orc.loss_and_grads(s, p, loss, x + h * u)[0] - orc.loss_and_grads(s, p, loss, x - h * u)[0]) / (2 * h)
    assert abs((g * u).sum() - fd) <= 1e-5 * abs(fd)


@pytest.mark.parametrize("form", ["lj", "dexp", "buck"])
def test_enthalpy_loss_direct_parameter_gradient(small_water, form):
    n_mol, box, x, _ = small_water
    s = orc.make_system(n_mol, box, form)
    p = np.array(C.default_params(form))
    loss = _ev_loss(s, x)
    l, _, _, dp = orc.loss_and_grads(s, p, loss, x)
    for k in range(len(p)):
        h = 1e-6 * abs(p[k])
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (orc.loss_and_grads(s, pp, loss, x)[0] - orc.loss_and_grads(s, pm, loss, x)[0]) / (2 * h)
        assert abs(dp[k] - fd) <= 1e-5 * max(abs(fd), 1e-3 * abs(l) / abs(p[k])), (k, dp[k], fd)


@pytest.mark.parametrize("rdf", [False, True])
def test_reverse_gradient_with_the_enthalpy_loss_matches_fd(small_water, rdf):
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    loss = _ev_loss(s, x, rdf)
    n = 20
    seeds = systems.noise_seeds(n, seed=4)
    xf, vf, lf, sx, sv, (fr, fe) = orc.forward_sim(s, p, x, v, seeds, 1.0, n, n, 0.001, loss, parts=True)
    assert abs(fr + fe - lf) <= 1e-12 * lf and fe > 0 and (fr > 0) == rdf
    _, _, lr, g, (rr, re) = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, n, n, 0.001, sx, sv, loss,
                                            parts=True)
    assert abs(lr - lf) <= 1e-9 * lf
    assert abs(re - fe) <= 1e-9 * fe
    fd = _fd_loss_grad(s, p, x, v, seeds, 1.0, n, loss)
    err = _scaled_err(g, fd, p)
    assert np.all(err < 3e-4), (err, g, fd)


def test_reverse_gradient_with_the_enthalpy_loss_multi_block(small_water):
    """Three loss blocks: the gradient is the mean of the per-block gradients, each the
    adjoint terms of its block plus the direct dl/dtheta at its loss point."""
    n_mol, box, x, v = small_water
    s = orc.make_system(n_mol, box)
    p = np.array(C.default_params())
    loss = _ev_loss(s, x, rdf=False)
    n, nl = 30, 10
    seeds = systems.noise_seeds(n, seed=5)
    xf, vf, lf, sx, sv = orc.forward_sim(s, p, x, v, seeds, 1.0, n, nl, 0.001, loss, n_steps_log=10)
    _, _, lr, g = orc.reverse_sim(s, p, xf, vf, seeds, 1.0, n, nl, nl, 0.001, sx, sv, loss, n_steps_log=10)
    assert abs(lr - lf) <= 1e-9 * lf
    fds = [_fd_loss_grad(s, p, sx[b].reshape(-1, 3), sv[b].reshape(-1, 3), seeds[b * nl:(b + 1) * nl],
                         1.0, nl, loss) for b in range(3)]
    err = _scaled_err(g, sum(fds) / 3, p)
    assert np.all(err < 3e-4), err
