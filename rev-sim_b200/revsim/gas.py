"""Gas diffusion in water: the host side of librevsim.so's gas-in-water engine
(include/revsim_gas.h) with the reference's diffusion/diffusion.jl entry points.

``GasEngine`` binds the C ABI.  ``forward_sim`` mirrors diffusion.jl:1181-1305 and
``reverse_sim`` diffusion.jl:1511-1616: same positional arguments, same meaning, same
return tuples.  Differences, each deliberate:

* coordinates / velocities are numpy arrays [N, 3] (nm, nm/ps), N = 3 n_water + 2 n_gas with
  the waters first (setup_system's order, diffusion.jl:1068-1118); ``coords_in=None`` (the
  reference's PDB start and steepest-descent minimisation) is not part of the engine;
* ``loss_type`` is any of diffusion.jl's :diff, :rdf, :ev, :diff_rdf, :diff_ev, :diff_rdf_ev
  (a leading ``:`` is accepted); the RDF term's targets are explicit (``loss_terms``, the
  engine's ``RdfTerm``s; ``loss.reference_rdf_terms`` builds the O-O / O-H L1 terms of
  diffusion.jl:759-774 from the Soper data the reference reads at load time, 673-686);
* ``run_grads=True`` (the Zygote unrolled-RAD check) is not part of the engine;
* the forward's snapshots and gas centres stay on the engine: ``sys.loggers`` is the engine
  and ``loss_accum`` carries the centres and the loss parts for inspection;
* ``n_threads`` is accepted and ignored; noise comes from the per-step seeds through the
  same counter-based Philox generator as the water engine.
"""

import ctypes

import numpy as np

from . import constants as C
from ._lib import GasDesc, RdfTermC, RevsimError, f64p, load, u64p

LOSS_BITS = {"diff": 1, "rdf": 2, "ev": 4, "diff_rdf": 3, "diff_ev": 5, "rdf_ev": 6,
             "diff_rdf_ev": 7}
INTER = {"lj": 0, "dexp": 1, "buck": 2, "ljsc": 3, "buff": 4}


def loss_bits(loss_type):
    lt = str(loss_type).lstrip(":")
    if lt in LOSS_BITS:
        return LOSS_BITS[lt]
    raise ValueError("loss_type not recognised")


class GasEngine:
    """One gas-in-water system on one GPU."""

    def __init__(self, n_water, n_gas, box, inter_type="lj", temp=C.TEMP, device=0,
                 precision="fp64", **consts):
        """precision: "fp64", or "mixed" for FP32 pair arithmetic (state, bonded terms,
        integrator, adjoints and sums stay FP64)."""
        self._h = None
        self._L = load()
        d = GasDesc()
        d.n_water, d.n_gas, d.box = int(n_water), int(n_gas), float(box)
        d.precision = {"fp64": 0, "mixed": 1}[precision]
        d.inter_type = INTER[inter_type] if isinstance(inter_type, str) else int(inter_type)
        d.temp = float(temp)
        d.device = int(device)
        for k, v in consts.items():
            setattr(d, k, v)
        h = ctypes.c_void_p()
        rc = self._L.revsim_gas_create(ctypes.byref(d), ctypes.byref(h))
        if rc:
            raise RevsimError(rc, "revsim_gas_create failed")
        self._h = h
        self.n_water, self.n_gas, self.box = int(n_water), int(n_gas), float(box)
        self.n_atoms = 3 * self.n_water + 2 * self.n_gas
        self.n_params = self._L.revsim_gas_n_params(d.inter_type)

    def _check(self, rc):
        if rc:
            msg = self._L.revsim_gas_last_error(self._h)
            raise RevsimError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_h", None):
            self._L.revsim_gas_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, theta):
        t = np.ascontiguousarray(theta, dtype=np.float64)
        self._check(self._L.revsim_gas_set_params(self._h, f64p(t), len(t)))

    def set_state(self, x, v):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.n_atoms, 3)
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(self.n_atoms, 3)
        self._check(self._L.revsim_gas_set_state(self._h, f64p(x), f64p(v)))

    def get_state(self):
        x, v = np.zeros((self.n_atoms, 3)), np.zeros((self.n_atoms, 3))
        self._check(self._L.revsim_gas_get_state(self._h, f64p(x), f64p(v)))
        return x, v

    def set_rdf(self, terms):
        """The RDF term's smoothed-RDF terms over the water atoms (engine.RdfTerm, one target
        [n_target] each); weighted 0.05 / n_blocks at every loss point."""
        terms = list(terms)
        arr = (RdfTermC * max(1, len(terms)))()
        tg = []
        for i, t in enumerate(terms):
            target = np.ascontiguousarray(t.target, dtype=np.float64).reshape(-1)
            tg.append(target)
            arr[i] = RdfTermC(t.sel1, t.sel2, t.x_min, t.step, t.width, t.exp_cutoff, t.n_grid,
                              t.slice_start, t.slice_stride, len(target), t.norm, t.weight)
        ptrs = (ctypes.POINTER(ctypes.c_double) * max(1, len(tg)))(*[f64p(a) for a in tg])
        self._check(self._L.revsim_gas_set_rdf(self._h, len(terms), arr, ptrs))
        self.rdf_terms = terms

    def forces(self):
        F = np.zeros((self.n_atoms, 3))
        self._check(self._L.revsim_gas_forces(self._h, f64p(F)))
        return F

    def force_vjp(self, w, acoef):
        """(F, dl_dfi, dl_dp) of calc_F_and_grads! against dl_dfi_prev = w and the
        contraction weights acoef."""
        w = np.ascontiguousarray(w, dtype=np.float64).reshape(self.n_atoms, 3)
        a = np.ascontiguousarray(acoef, dtype=np.float64).reshape(self.n_atoms, 3)
        F, G, dp = np.zeros((self.n_atoms, 3)), np.zeros((self.n_atoms, 3)), np.zeros(self.n_params)
        self._check(self._L.revsim_gas_force_vjp(self._h, f64p(w), f64p(a), f64p(F), f64p(G), f64p(dp)))
        return F, G, dp

    def energy(self, grads=False):
        E = ctypes.c_double()
        dp = np.zeros(self.n_params)
        self._check(self._L.revsim_gas_energy(self._h, ctypes.byref(E), f64p(dp) if grads else None))
        return (E.value, dp) if grads else E.value

    def forward(self, seeds, gamma, n_steps, n_steps_loss, dt, loss_type="diff", calc_loss=True):
        """(loss, [D m^2/s, l_diff, l_rdf, l_ev], centres [n_blocks, n_gas, 3])."""
        bits = loss_bits(loss_type)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        nb = n_steps // n_steps_loss if n_steps else 0
        centres = np.zeros((nb, self.n_gas, 3))
        loss = ctypes.c_double()
        parts = np.zeros(4)
        self._check(self._L.revsim_gas_forward(self._h, u64p(seeds), float(gamma), int(n_steps),
                                               int(n_steps_loss), float(dt), bits,
                                               1 if calc_loss else 0, ctypes.byref(loss),
                                               f64p(parts), f64p(centres)))
        return loss.value, parts, centres

    def reverse(self, seeds, gamma, n_steps, n_steps_loss, n_steps_trunc, dt, loss_type="diff"):
        """(loss, dl_dp, [D m^2/s, l_diff, l_rdf, l_ev])."""
        bits = loss_bits(loss_type)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        loss = ctypes.c_double()
        g, parts = np.zeros(self.n_params), np.zeros(4)
        self._check(self._L.revsim_gas_reverse(self._h, u64p(seeds), float(gamma), int(n_steps),
                                               int(n_steps_loss), int(n_steps_trunc), float(dt),
                                               bits, ctypes.byref(loss), f64p(g), f64p(parts)))
        return loss.value, g, parts

    def stream(self):
        return self._L.revsim_gas_stream(self._h)

    def launch_count(self):
        return int(self._L.revsim_gas_launch_count(self._h))

    def set_kernel_timing(self, on):
        self._check(self._L.revsim_gas_set_kernel_timing(self._h, 1 if on else 0))

    def kernel_time(self, which):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        self._check(self._L.revsim_gas_kernel_time(self._h, int(which), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value


class GasSystem:
    """What forward_sim / reverse_sim return in place of Molly's System."""

    def __init__(self, engine, coords, velocities):
        self.engine = engine
        self.coords = coords
        self.velocities = velocities
        self.boundary = engine.box

    @property
    def loggers(self):
        return self.engine


class LossAccum:
    """loss_accum of diffusion.jl:817-821: the gas centres of every loss point and the loss
    parts (D in m^2/s, l_diff, l_rdf, l_ev)."""

    def __init__(self, gas_coords, parts):
        self.gas_coords = gas_coords
        self.D, self.l_diff, self.l_rdf, self.l_ev = (float(p) for p in parts)


def _engine_for(coords, inter_type, engine, n_gas, box):
    n_atoms = np.asarray(coords).shape[0]
    if engine is not None:
        if engine.n_atoms != n_atoms:
            raise ValueError("coords do not match the engine's system")
        return engine
    if n_atoms < 2 * n_gas or (n_atoms - 2 * n_gas) % 3:
        raise ValueError("coords must hold 3 n_water + 2 n_gas atoms")
    return GasEngine((n_atoms - 2 * n_gas) // 3, n_gas, box, inter_type)


def forward_sim(coords_in, velocities_in, noise_seeds, gamma, n_steps, n_steps_loss, params, dt,
                n_threads, inter_type, loss_type, run_grads=False, calc_loss=True, *, engine=None,
                n_gas=C.GAS_N_GAS, box=C.GAS_BOX, loss_terms=None):
    """diffusion.jl:1181.  Returns (sys, loss, loss_accum, grads); grads is [None] * P as in
    the reference's run_grads=false branch (diffusion.jl:1301-1303)."""
    if run_grads:
        raise NotImplementedError("run_grads (Zygote unrolled RAD) is not part of the engine")
    if coords_in is None or velocities_in is None:
        raise ValueError("the engine starts from given coordinates and velocities")
    eng = _engine_for(coords_in, inter_type, engine, n_gas, box)
    if loss_terms is not None:
        eng.set_rdf(loss_terms)
    eng.set_params(params)
    eng.set_state(coords_in, velocities_in)
    loss, parts, centres = eng.forward(noise_seeds, gamma, n_steps, n_steps_loss, dt, loss_type,
                                       calc_loss)
    x, v = eng.get_state()
    return GasSystem(eng, x, v), loss, LossAccum(centres, parts), [None] * eng.n_params


def reverse_sim(coords, velocities, noise_seeds, gamma, n_steps, n_steps_loss, n_steps_trunc,
                params, dt, n_threads, fwd_loggers, loss_accum_fwd, inter_type, loss_type):
    """diffusion.jl:1511.  ``fwd_loggers`` is ``sys.loggers`` of the forward_sim result (the
    engine holding the snapshots and centres; the reference also restarts from its last
    snapshot, diffusion.jl:1557-1558).  Returns (sys, loss, dl_dp, D, l_diff, l_rdf, l_ev)
    with D in m^2/s."""
    eng = fwd_loggers
    if not isinstance(eng, GasEngine):
        raise TypeError("fwd_loggers must be the loggers of a forward_sim result")
    eng.set_params(params)
    loss, g, parts = eng.reverse(noise_seeds, gamma, n_steps, n_steps_loss, n_steps_trunc, dt,
                                 loss_type)
    x, v = eng.get_state()
    return (GasSystem(eng, x, v), loss, g, float(parts[0]), float(parts[1]), float(parts[2]),
            float(parts[3]))
