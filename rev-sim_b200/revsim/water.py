"""The reference's gradient entry points, with the reference's signatures.

``forward_sim`` mirrors water.jl:977-1105, ``reverse_sim`` water.jl:1435-1558 and
``reweighting_sim`` water.jl:1107-1210:
same positional arguments, same meaning, same return tuples, so a caller of the
reference (the self-check block water.jl:1592-1621, ``train()`` water.jl:1662-1669)
switches by changing the import.  The work runs in librevsim.so on the GPU.

Differences, each deliberate:
* coordinates/velocities are numpy arrays [N, 3] (nm, nm/ps); ``boundary`` is the
  cubic box side in nm (``None``: keep the engine's);
* the loss targets are explicit (``loss_terms``): the reference reads the Soper
  2013 file at load time (water.jl:629); ``loss.read_rdf_data`` + ``loss.reference_rdf_terms``
  rebuild exactly that loss from the file;
* ``loss_type`` is ``"rdf"``, ``"enth_vap"`` or ``"both"`` as in loss_fn (water.jl:757-769);
  the RDF terms stay on the engine between calls, so ``loss_terms`` is needed once;
* ``use_barostat=True`` runs the engine's Monte-Carlo barostat (its draws from a stream keyed
  by the first noise seed; the returned ``sys.boundary`` is the final box); ``run_grads=True``
  (the Zygote unrolled-RAD check, water.jl:1052-1099) is not part of the engine and raises
  ``NotImplementedError``;
* ``n_threads`` is accepted and ignored;
* noise: per-step seeds drive a counter-based Philox generator, regenerated
  identically in the reverse pass (the reference uses Xoshiro(seed) + randn); a caller
  that holds the reference's own noise (generate_noise!, water.jl:867-873, one [N, 3] array
  per step) passes it as ``host_noise`` [n_steps, N, 3] to both calls instead, and the
  engine then integrates exactly the reference's trajectory.
"""

import numpy as np

from . import constants as C
from .engine import Engine


class SimSystem:
    """What forward_sim / reverse_sim return in place of Molly's System."""

    def __init__(self, engine, coords, velocities, boundary):
        self.engine = engine
        self.coords = coords
        self.velocities = velocities
        self.boundary = boundary

    @property
    def loggers(self):
        # The forward snapshots (every n_steps_log steps) and neighbour-build positions
        # live on the device inside the engine; reverse_sim takes the engine itself.
        return self.engine


def _engine_for(coords, boundary, inter_type, engine, precision):
    n_atoms = np.asarray(coords).shape[0]
    if n_atoms % 3:
        raise ValueError("water systems have 3 atoms per molecule")
    if engine is not None:
        if boundary is not None and not np.array_equal(np.broadcast_to(boundary, engine.box.shape),
                                                       engine.box):
            engine.set_box(boundary)   # the boundary argument (water.jl:1001)
        return engine
    return Engine(n_atoms // 3, boundary, inter_type=inter_type, precision=precision)


LOSS_TYPES = {"rdf": (True, False), "enth_vap": (False, True), "both": (True, True)}


def _set_loss(eng, loss_type, loss_terms):
    """loss_fn's loss_type (water.jl:757-769): the RDF terms, the enthalpy term, or both."""
    loss_type = str(loss_type).lstrip(":")
    if loss_type not in LOSS_TYPES:
        raise ValueError("loss_type not recognised")
    use_rdf, use_ev = LOSS_TYPES[loss_type]
    if loss_terms is not None:
        eng.rdf_terms = list(loss_terms)
    if use_rdf and not eng.rdf_terms:
        raise ValueError(f"loss_type {loss_type!r} needs loss_terms")
    eng.set_loss(eng.rdf_terms if use_rdf else [])
    eng.set_enth_vap(use_ev)


def forward_sim(coords, velocities, boundary, noise_seeds, gamma, n_steps, n_steps_loss, params,
                dt, n_threads, inter_type, loss_type, run_grads=False, calc_loss=True,
                use_barostat=False, *, loss_terms=None, engine=None, precision="fp64",
                host_noise=None):
    """water.jl:977.  Returns (sys, loss, grads); grads is [None] * P as in the
    reference's run_grads=false branch (water.jl:1100-1102).  ``host_noise``
    [n_steps, N, 3]: the noise of every step, used in place of the seeds' draws."""
    if run_grads:
        raise NotImplementedError("run_grads (Zygote unrolled RAD) is not part of the engine")
    eng = _engine_for(coords, boundary, inter_type, engine, precision)
    eng.set_params(params)
    eng.set_state(coords, velocities)
    if calc_loss:
        _set_loss(eng, loss_type, loss_terms)
    seeds = np.asarray(noise_seeds, dtype=np.uint64)
    if use_barostat:
        # MonteCarloBarostatNoUnits(1 bar, temp, boundary) (water.jl:1009-1014); its draws
        # come from a stream keyed by the run's first noise seed
        eng.set_barostat(True, seed=int(seeds.reshape(-1)[0]) if seeds.size else 0)
    try:
        loss = eng.forward(seeds, gamma, n_steps, n_steps_loss if n_steps_loss else max(n_steps, 1),
                           dt, calc_loss, noise=host_noise)
    finally:
        if use_barostat:
            eng.set_barostat(False)
    x, v = eng.get_state()
    box = eng.barostat_state()[0]
    sys = SimSystem(eng, x, v, float(box[0]) if eng.R == 1 else box)
    return sys, (float(loss[0]) if eng.R == 1 else loss), [None] * eng.n_params


def reverse_sim(coords, velocities, boundary, noise_seeds, gamma, n_steps, n_steps_loss,
                n_steps_trunc, params, dt, n_threads, fwd_loggers, clip_norm_threshold, inter_type,
                loss_type, *, loss_terms=None, host_noise=None):
    """water.jl:1435.  ``fwd_loggers`` is ``sys.loggers`` of the forward_sim result;
    ``host_noise`` the array the forward_sim call was given, if any.
    Returns (sys, l, dl_dp, l_rdf, l_ev)."""
    if n_steps_trunc > n_steps_loss:
        raise ValueError("n_steps_trunc must not be greater than n_steps_loss")
    eng = fwd_loggers
    if not isinstance(eng, Engine):
        raise TypeError("fwd_loggers must be the loggers of a forward_sim result")
    _set_loss(eng, loss_type, loss_terms)
    eng.set_params(params)
    eng.set_state(coords, velocities)
    clip = np.inf if clip_norm_threshold is None else float(clip_norm_threshold)
    loss, g = eng.reverse(noise_seeds, gamma, n_steps, n_steps_loss, n_steps_trunc, dt, clip,
                          noise=host_noise)
    x, v = eng.get_state()
    sys = SimSystem(eng, x, v, float(eng.box[0]) if boundary is None else boundary)
    l_rdf, l_ev = eng.loss_parts()
    if eng.R == 1:
        return sys, float(loss[0]), g[0], float(l_rdf[0]), float(l_ev[0])
    return sys, loss, g, l_rdf, l_ev


def reweighting_sim(coords, velocities, boundary, noise_seeds, gamma, n_steps, n_steps_loss, params,
                    dt, n_threads, inter_type, loss_type, use_barostat=False, *, loss_terms=None,
                    engine=None, precision="fp64", temp=C.TEMP):
    """water.jl:1107-1210: the ensemble-reweighting gradient estimator,
    dL/dtheta = <dl/dtheta> - beta (<L dE/dtheta> - <L> <dE/dtheta>), averages over the loss
    points (every n_steps_loss steps) of one forward run, beta = 1 / (k_B T); dl/dtheta is the
    enthalpy term's direct gradient (zero for the RDF loss).  Returns
    (sys, loss, grads, l_rdf, l_ev)."""
    eng = _engine_for(coords, boundary, inter_type, engine, precision)
    eng.set_params(params)
    eng.set_state(coords, velocities)
    _set_loss(eng, loss_type, loss_terms)
    seeds = np.asarray(noise_seeds, dtype=np.uint64)
    if use_barostat:
        # one barostat over the whole run: its step count carries across the blocks
        eng.set_barostat(True, seed=int(seeds.reshape(-1)[0]) if seeds.size else 0)
    n_blocks = 1 if n_steps == 0 else n_steps // n_steps_loss
    acc = np.zeros((3, eng.R))   # loss, l_rdf, l_ev
    dl_acc = np.zeros((eng.R, eng.n_params))
    dE_acc = np.zeros((eng.R, eng.n_params))
    l_dE_acc = np.zeros((eng.R, eng.n_params))
    for b in range(n_steps // n_steps_loss):
        # the forward run in blocks of n_steps_loss; loss_and_grads at each block's end is the
        # reference's at step_n % n_steps_loss == 0 (water.jl:1176)
        eng.forward(seeds[b * n_steps_loss:(b + 1) * n_steps_loss], gamma, n_steps_loss,
                    n_steps_loss, dt, calc_loss=False)
        lb, lrb, leb, _, dlb = eng.loss_and_grads()
        _, dE = eng.energy_grad()
        acc += np.stack([lb, lrb, leb])
        dl_acc += dlb
        dE_acc += dE
        l_dE_acc += lb[:, None] * dE
    if use_barostat:
        eng.set_barostat(False)
    loss, l_rdf, l_ev = acc / n_blocks
    beta = 1.0 / (C.KB * np.asarray(temp, dtype=np.float64))
    beta = np.broadcast_to(beta, (eng.R,))[:, None]
    grads = dl_acc / n_blocks - beta * (l_dE_acc / n_blocks - loss[:, None] * dE_acc / n_blocks)
    x, v = eng.get_state()
    sys = SimSystem(eng, x, v, float(eng.box[0]) if boundary is None else boundary)
    if eng.R == 1:
        return sys, float(loss[0]), grads[0], float(l_rdf[0]), float(l_ev[0])
    return sys, loss, grads, l_rdf, l_ev


def default_params(inter_type="lj"):
    return np.array(C.default_params(inter_type))
