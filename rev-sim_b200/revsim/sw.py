"""SwEngine: an owning Python wrapper of one revsim_sw_handle (Stillinger-Weber diamond),
and the reference's diamond ``forward_sim`` / ``reverse_sim`` entry points on top of it.

Mirrors greener-group/rev-sim ``diamond/diamond.jl`` for inter_type :sw and loss_type
:stress: ``forward_sim`` (diamond.jl:1394-1538) and ``reverse_sim`` (diamond.jl:1757-1878)
keep their argument order and meaning; the loggers the reference hands from the forward to
the reverse pass (the states at the loss points) stay on the device inside the engine.
"""

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import diamond as D
from ._lib import RevsimError, as_f64, f64p, u64p

PRECISION = {"fp64": 0, "mixed": 1}


class SwEngine:
    """Device state for R diamond replicas (n_atoms, box, temp: scalars or per replica)."""

    def __init__(self, n_atoms, box, temp=D.TEMP, precision="mixed", device=0, skin=0.05,
                 n_steps_nf=10, mass=D.C_MASS, mlp=False):
        self._L = _lib.load()
        n_atoms = np.atleast_1d(np.asarray(n_atoms, dtype=np.int32))
        R = len(n_atoms)
        self.n_atoms = n_atoms
        self.box = np.broadcast_to(np.asarray(box, dtype=np.float64), (R,)).copy()
        self.temp = np.broadcast_to(np.asarray(temp, dtype=np.float64), (R,)).copy()
        self.R, self.N = R, int(n_atoms.sum())
        self.precision = precision
        self.mass = mass
        self.mlp = bool(mlp)
        # the 7 SW parameters, then the learned radial term's (one MLP type)
        self.n_params = D.N_PARAMS + (D.MLP_NPARAMS if mlp else 0)
        desc = _lib.SwDesc(R, n_atoms.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                           f64p(self.box), f64p(self.temp), PRECISION[precision], mass, D.KB,
                           skin, n_steps_nf, device, 1 if mlp else 0)
        h = ctypes.c_void_p()
        rc = self._L.revsim_sw_create(ctypes.byref(desc), ctypes.byref(h))
        if rc != 0:
            raise RevsimError(rc, "revsim_sw_create failed")
        self._h = h

    # ------------------------------------------------------------------ plumbing
    def _ck(self, rc):
        if rc != 0:
            raise RevsimError(rc, self._L.revsim_sw_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.revsim_sw_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _vec(self, a):
        return as_f64(a, (self.N, 3))

    # ---------------------------------------------------------------- interface
    def set_params(self, theta):
        t = as_f64(theta)
        self._ck(self._L.revsim_sw_set_params(self._h, f64p(t), len(t)))

    def set_state(self, x, v):
        x, v = self._vec(x), self._vec(v)
        self._ck(self._L.revsim_sw_set_state(self._h, f64p(x), f64p(v)))

    def get_state(self):
        x = np.zeros((self.N, 3))
        v = np.zeros((self.N, 3))
        self._ck(self._L.revsim_sw_get_state(self._h, f64p(x), f64p(v)))
        return x, v

    def set_loss(self, weight=D.STRESS_WEIGHT, target=None, vel_term=True):
        t = np.zeros((self.R, 9)) if target is None else as_f64(
            np.broadcast_to(np.asarray(target, dtype=np.float64).reshape(-1, 9), (self.R, 9)))
        self._loss_target = np.ascontiguousarray(t)
        L = _lib.SwLossC(weight, 1 if vel_term else 0, f64p(self._loss_target))
        self._ck(self._L.revsim_sw_set_loss(self._h, ctypes.byref(L)))

    def set_lanes(self, lanes):
        self._ck(self._L.revsim_sw_set_lanes(self._h, int(lanes)))

    def forces(self):
        F = np.zeros((self.N, 3))
        self._ck(self._L.revsim_sw_forces(self._h, f64p(F)))
        return F

    def force_vjp(self, w, acoef=None):
        """(F, dl_dfi = sum_a (w_a/m) dF_a/dx, dtheta[R, n_params] = sum_a acoef_a dF_a/dtheta)."""
        w = self._vec(w)
        a = None if acoef is None else self._vec(acoef)
        F = np.zeros((self.N, 3))
        G = np.zeros((self.N, 3))
        dth = np.zeros((self.R, self.n_params))
        self._ck(self._L.revsim_sw_force_vjp(self._h, f64p(w), f64p(a) if a is not None else None,
                                             f64p(F), f64p(G), f64p(dth)))
        return F, G, (dth if a is not None else None)

    def stress(self, vel_term=True):
        s = np.zeros((self.R, 9))
        self._ck(self._L.revsim_sw_stress(self._h, 1 if vel_term else 0, f64p(s)))
        return s.reshape(self.R, 3, 3)

    def loss_grad(self):
        """(loss[R], dL/dx [N, 3], dL/dv [N, 3], dL/dtheta [R, n_params]) at the current state."""
        loss = np.zeros(self.R)
        gx = np.zeros((self.N, 3))
        gv = np.zeros((self.N, 3))
        gp = np.zeros((self.R, self.n_params))
        self._ck(self._L.revsim_sw_loss_grad(self._h, f64p(loss), f64p(gx), f64p(gv), f64p(gp)))
        return loss, gx, gv, gp

    def noise(self, seeds):
        s = np.ascontiguousarray(np.broadcast_to(np.asarray(seeds, dtype=np.uint64), (self.R,)))
        xi = np.zeros((self.N, 3))
        self._ck(self._L.revsim_sw_noise(self._h, u64p(s), f64p(xi)))
        return xi

    def active_pairs(self):
        """Sorted [n, 2] array of global atom indices i < j with r / sigma < a."""
        n = ctypes.c_int64()
        self._ck(self._L.revsim_sw_active_pairs(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros((max(n.value, 1), 2), dtype=np.int32)
        self._ck(self._L.revsim_sw_active_pairs(
            self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), n.value, ctypes.byref(n)))
        out = out[:n.value]
        return out[np.lexsort((out[:, 1], out[:, 0]))]

    def _seeds(self, seeds, n_steps):
        s = np.asarray(seeds, dtype=np.uint64)
        if s.ndim == 1:
            s = np.repeat(s[:, None], self.R, axis=1)
        return np.ascontiguousarray(s.reshape(n_steps, self.R))

    def forward(self, seeds, gamma, n_steps, n_steps_loss, dt, n_steps_buffer=0, calc_loss=True):
        """Forward pass; returns (loss[R], n_blocks).  seeds: [n_steps] or [n_steps, R]."""
        s = self._seeds(seeds, n_steps)
        loss = np.zeros(self.R)
        nb = ctypes.c_int32()
        self._ck(self._L.revsim_sw_forward(self._h, u64p(s), gamma, n_steps, n_steps_loss,
                                           n_steps_buffer, dt, 1 if calc_loss else 0, f64p(loss),
                                           ctypes.byref(nb)))
        return loss, nb.value

    def reverse(self, seeds, gamma, n_steps, n_steps_loss, n_steps_trunc, dt):
        """Reverse pass from the forward end state; returns (loss[R], dL/dtheta [R, n_params])."""
        s = self._seeds(seeds, n_steps)
        loss = np.zeros(self.R)
        g = np.zeros((self.R, self.n_params))
        self._ck(self._L.revsim_sw_reverse(self._h, u64p(s), gamma, n_steps, n_steps_loss,
                                           n_steps_trunc, dt, f64p(loss), f64p(g)))
        return loss, g

    def launch_count(self):
        n = ctypes.c_int64()
        self._ck(self._L.revsim_sw_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def set_kernel_timing(self, on=True):
        self._ck(self._L.revsim_sw_set_kernel_timing(self._h, 1 if on else 0))

    def kernel_time(self, which):
        """which: 0 reverse terms, 1 forward terms, 2 reverse gather, 3 forward gather."""
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        self._ck(self._L.revsim_sw_kernel_time(self._h, which, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def stream(self):
        p = ctypes.c_void_p()
        self._ck(self._L.revsim_sw_stream(self._h, ctypes.byref(p)))
        return p.value


# ------------------------------------------------------------------------------------
# The reference's entry points (diamond.jl), :sw interaction with the :stress loss.

@dataclass
class SwSystem:
    """What forward_sim / reverse_sim hand back in place of a Molly System: the state and
    the engine that keeps the forward pass's loss-point states for the reverse pass."""
    coords: np.ndarray
    velocities: np.ndarray
    loggers: object = None


def _engine_for(coords, box, precision, engine, mlp):
    if engine is not None:
        return engine
    n = len(np.asarray(coords).reshape(-1, 3))
    return SwEngine(n, box, precision=precision, mlp=mlp)


def _theta(eng, params_sw, params_gnn):
    """The engine's parameter vector: the SW parameters, then -- with the learned term, which
    stands in for the reference's GNN -- params_gnn."""
    if eng.mlp:
        if params_gnn is None:
            raise ValueError("an engine with the learned term needs params_gnn (its MLP parameters)")
        return np.concatenate([np.asarray(params_sw, dtype=np.float64), np.asarray(params_gnn, dtype=np.float64)])
    return np.asarray(params_sw, dtype=np.float64)


def forward_sim(coords_in, velocities_in, noise_seeds, gamma, n_steps, n_steps_loss,
                n_steps_buffer, params_sw, params_gnn, dt, n_threads=1, inter_type="sw",
                loss_type="stress", run_grads=False, calc_loss=True, *, box=D.SIDE_LENGTH,
                precision="mixed", engine=None, weight=D.STRESS_WEIGHT, target=None):
    """diamond.jl:1394-1538 for :sw / :stress.  Returns (sys, loss, loss_accum_blocks,
    loss_logs, grads_sw, grads_gnn); ``run_grads`` (the forward-mode AD check of the
    reference) is not available and must be False; params_gnn holds the learned radial term's
    MLP parameters (None: no learned term)."""
    if inter_type != "sw" or loss_type != "stress":
        raise ValueError("the engine implements inter_type :sw with loss_type :stress")
    if run_grads:
        raise ValueError("run_grads (forward-mode AD through the whole run) is not provided; "
                         "use reverse_sim")
    eng = _engine_for(coords_in, box, precision, engine, params_gnn is not None)
    eng.set_params(_theta(eng, params_sw, params_gnn))
    eng.set_state(coords_in, velocities_in)
    eng.set_loss(weight, target)
    loss, nb = eng.forward(noise_seeds, gamma, n_steps, n_steps_loss, dt, n_steps_buffer,
                           calc_loss)
    x, v = eng.get_state()
    sys = SwSystem(x, v, eng)
    l = float(loss.mean()) if calc_loss else 0.0
    return (sys, l, {"stress": l * nb, "n_blocks": nb}, {"stress": l}, np.zeros(D.N_PARAMS),
            np.zeros(D.MLP_NPARAMS) if eng.mlp else None)


def reverse_sim(coords, velocities, noise_seeds, gamma, n_steps, n_steps_loss, n_steps_trunc,
                n_steps_buffer, params_sw, params_gnn, dt, n_threads, fwd_loggers, loss_accum_fwd,
                inter_type="sw", loss_type="stress"):
    """diamond.jl:1757-1878 for :sw / :stress: (sys, loss, dl_dp_sw, dl_dp_gnn).
    ``fwd_loggers`` is the engine returned as ``sys.loggers`` by forward_sim."""
    if inter_type != "sw" or loss_type != "stress":
        raise ValueError("the engine implements inter_type :sw with loss_type :stress")
    eng = fwd_loggers
    if not isinstance(eng, SwEngine):
        raise ValueError("fwd_loggers must be the engine returned by forward_sim")
    # the forward record stays valid for unchanged parameters
    eng.set_params(_theta(eng, params_sw, params_gnn))
    eng.set_state(coords, velocities)
    loss, g = eng.reverse(noise_seeds, gamma, n_steps, n_steps_loss, n_steps_trunc, dt)
    x, v = eng.get_state()
    g = g.mean(axis=0)
    return (SwSystem(x, v, eng), float(loss.mean()), g[:D.N_PARAMS],
            g[D.N_PARAMS:] if eng.mlp else None)
