"""Engine: an owning Python wrapper of one revsim_handle (one or more water replicas)."""

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import constants as C
from ._lib import RevsimError, as_f64, f64p, u64p

PRECISION = {"fp64": 0, "mixed": 1}
NL_MODE = {"checkpoint": 0, "reconstructed": 1}


@dataclass
class RdfTerm:
    """One smoothed-RDF loss term (revsim_rdf_term).  sel: 0 = O, 1 = H.
    ``target`` is [n_target] (shared by all replicas) or [n_replicas, n_target]."""
    sel1: int
    sel2: int
    x_min: float
    step: float
    width: float
    exp_cutoff: float
    n_grid: int
    slice_start: int
    slice_stride: int
    target: np.ndarray
    norm: int = 2
    weight: float = 1.0


class Engine:
    """Owns device state for R replicas of a flexible 3-site water box.

    n_mol, box, temp: scalars (one replica) or sequences (one entry per replica).
    """

    def __init__(self, n_mol, box, temp=C.TEMP, inter_type="lj", precision="fp64",
                 nl_mode="checkpoint", device=0, n_steps_log=C.N_STEPS_LOG,
                 n_steps_nf=C.N_STEPS_NF, cutoff=C.DIST_CUTOFF, nl_cutoff=C.DIST_NEIGHBORS,
                 coulomb_const=C.COULOMB_CONST, crf_const=None, mlp=False):
        self._L = _lib.load()
        n_mol = np.atleast_1d(np.asarray(n_mol, dtype=np.int32))
        R = len(n_mol)
        box = np.broadcast_to(np.asarray(box, dtype=np.float64), (R,)).copy()
        temp = np.broadcast_to(np.asarray(temp, dtype=np.float64), (R,)).copy()
        if crf_const is None:
            crf_const = (1.0 / cutoff**3) * ((78.3 - 1) / (2 * 78.3 + 1))
        self.n_mol, self.box, self.temp = n_mol, box, temp
        self.R = R
        self.inter_type = inter_type
        self.precision = precision
        self.mlp = bool(mlp)
        self._keep = (n_mol, box, temp)
        desc = _lib.SystemDesc(
            R, n_mol.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), f64p(box), f64p(temp),
            C.INTER_TYPES[inter_type], PRECISION[precision], C.O_MASS, C.H_MASS, coulomb_const,
            crf_const, cutoff, nl_cutoff, C.KB, n_steps_nf, n_steps_log, NL_MODE[nl_mode], device,
            1 if mlp else 0)
        h = ctypes.c_void_p()
        rc = self._L.revsim_create(ctypes.byref(desc), ctypes.byref(h))
        if rc != 0:
            raise RevsimError(rc, "revsim_create failed (bad description or no CUDA device)")
        self._h = h
        n_atoms = ctypes.c_int64()
        n_params = ctypes.c_int32()
        self._check(self._L.revsim_sizes(h, ctypes.byref(n_atoms), ctypes.byref(n_params)))
        self.n_atoms = n_atoms.value
        self.n_params = n_params.value
        self.atom0 = np.concatenate([[0], np.cumsum(3 * n_mol)[:-1]]).astype(np.int64)
        self.terms = []
        self.rdf_terms = []      # the RDF terms loss_type :rdf / :both use (water.py)
        self.enth_vap = False

    # ------------------------------------------------------------------ basics
    def _check(self, rc):
        if rc != 0:
            msg = self._L.revsim_last_error(self._h).decode() if getattr(self, "_h", None) else ""
            raise RevsimError(rc, msg)

    def close(self):
        if getattr(self, "_h", None):
            self._L.revsim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def stream(self):
        return self._L.revsim_stream(self._h)

    def launch_count(self):
        return self._L.revsim_launch_count(self._h)

    # ------------------------------------------------------------------ state
    def set_params(self, theta):
        theta = as_f64(theta)
        self._check(self._L.revsim_set_params(self._h, f64p(theta), len(theta)))

    def set_state(self, x, v):
        x = as_f64(x, (self.n_atoms, 3))
        v = as_f64(v, (self.n_atoms, 3))
        self._check(self._L.revsim_set_state(self._h, f64p(x), f64p(v)))

    def get_state(self):
        x = np.zeros((self.n_atoms, 3))
        v = np.zeros((self.n_atoms, 3))
        self._check(self._L.revsim_get_state(self._h, f64p(x), f64p(v)))
        return x, v

    def set_loss(self, terms):
        self.terms = list(terms)
        arr = (_lib.RdfTermC * max(1, len(terms)))()
        tg = []
        for i, t in enumerate(terms):
            target = np.asarray(t.target, dtype=np.float64)
            if target.ndim == 1:
                target = np.broadcast_to(target, (self.R, target.size))
            target = np.ascontiguousarray(target)
            tg.append(target)
            arr[i] = _lib.RdfTermC(t.sel1, t.sel2, t.x_min, t.step, t.width, t.exp_cutoff,
                                   t.n_grid, t.slice_start, t.slice_stride, target.shape[1],
                                   t.norm, t.weight)
        ptrs = (ctypes.POINTER(ctypes.c_double) * max(1, len(tg)))(*[f64p(a) for a in tg])
        self._check(self._L.revsim_set_loss(self._h, len(terms), arr, ptrs))

    # ------------------------------------------------------------ primitives
    def forces(self):
        F = np.zeros((self.n_atoms, 3))
        self._check(self._L.revsim_forces(self._h, f64p(F)))
        return F

    def force_vjp(self, w, acoef):
        w = as_f64(w, (self.n_atoms, 3))
        acoef = as_f64(acoef, (self.n_atoms, 3))
        F = np.zeros((self.n_atoms, 3))
        G = np.zeros((self.n_atoms, 3))
        th = np.zeros((self.R, self.n_params))
        self._check(self._L.revsim_force_vjp(self._h, f64p(w), f64p(acoef), f64p(F), f64p(G),
                                             f64p(th)))
        return F, G, th

    def energy_grad(self):
        """(E [R], dE/dtheta [R, n_params]) at the current state."""
        E = np.zeros(self.R)
        g = np.zeros((self.R, self.n_params))
        self._check(self._L.revsim_energy_grad(self._h, f64p(E), f64p(g)))
        return E, g

    def noise(self, seeds):
        seeds = np.ascontiguousarray(np.broadcast_to(np.asarray(seeds, dtype=np.uint64), (self.R,)))
        xi = np.zeros((self.n_atoms, 3))
        self._check(self._L.revsim_noise(self._h, u64p(seeds), f64p(xi)))
        return xi

    def neighbor_pairs(self, replica=0):
        n = ctypes.c_int64()
        cap = 400 * 3 * int(self.n_mol[replica]) + 64
        out = np.zeros((cap, 2), dtype=np.int32)
        pi = out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        self._check(self._L.revsim_neighbor_pairs(self._h, replica, pi, cap, ctypes.byref(n)))
        if n.value > cap:
            cap = n.value
            out = np.zeros((cap, 2), dtype=np.int32)
            pi = out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            self._check(self._L.revsim_neighbor_pairs(self._h, replica, pi, cap, ctypes.byref(n)))
        p = out[: n.value]
        return p[np.lexsort((p[:, 1], p[:, 0]))]

    def loss_grad(self, grad=True):
        loss = np.zeros(self.R)
        g = np.zeros((self.n_atoms, 3)) if grad else None
        self._check(self._L.revsim_loss_grad(self._h, f64p(loss), f64p(g) if grad else None))
        return loss, g

    def set_barostat(self, enable=True, pressure=1.0, n_steps=30, scale_factor=0.01,
                     scale_increment=1.1, max_volume_frac=0.3, seed=0):
        """Monte-Carlo barostat of forward passes (MonteCarloBarostatNoUnits, water.jl:789-865,
        with its defaults of water.jl:802-806); enable=False switches it off."""
        if not enable:
            self._check(self._L.revsim_set_barostat(self._h, None))
            return
        d = _lib.BarostatDesc(pressure, n_steps, scale_factor, scale_increment, max_volume_frac,
                              int(seed) & 0xFFFFFFFFFFFFFFFF)
        self._check(self._L.revsim_set_barostat(self._h, ctypes.byref(d)))

    def barostat_state(self):
        """(box [R], volume_scale [R], attempts [R], accepted [R])."""
        box, vs = np.zeros(self.R), np.zeros(self.R)
        na, nacc = np.zeros(self.R, dtype=np.int64), np.zeros(self.R, dtype=np.int64)
        p64 = ctypes.POINTER(ctypes.c_int64)
        self._check(self._L.revsim_barostat_state(self._h, f64p(box), f64p(vs), na.ctypes.data_as(p64),
                                                  nacc.ctypes.data_as(p64)))
        self.box = box.copy()
        return box, vs, na, nacc

    def set_box(self, box):
        """New cubic box sides [R] (the boundary argument of forward_sim / reverse_sim)."""
        b = np.ascontiguousarray(np.broadcast_to(np.asarray(box, dtype=np.float64), (self.R,)))
        self._check(self._L.revsim_set_box(self._h, f64p(b)))
        self.box = b.copy()

    def set_enth_vap(self, enable=True, u_gas=C.ENTH_U_GAS, rt=C.ENTH_RT, target=C.ENTH_TARGET):
        """Add (or with enable=False remove) the enthalpy-of-vaporisation loss term
        (loss_enth_vap, water.jl:738-755) to the RDF terms of set_loss."""
        self._check(self._L.revsim_set_enth_vap(self._h, 1 if enable else 0, u_gas, rt, target))
        self.enth_vap = bool(enable)

    def loss_parts(self):
        """(l_rdf [R], l_ev [R]) of the loss the last forward / reverse returned."""
        lr, le = np.zeros(self.R), np.zeros(self.R)
        self._check(self._L.revsim_loss_parts(self._h, f64p(lr), f64p(le)))
        return lr, le

    def loss_and_grads(self):
        """loss_and_grads (water.jl:771-786) at the current state: (loss [R], l_rdf [R],
        l_ev [R], dL/dx [N, 3], direct dl/dtheta [R, n_params])."""
        out = [np.zeros(self.R) for _ in range(3)]
        g = np.zeros((self.n_atoms, 3))
        dp = np.zeros((self.R, self.n_params))
        self._check(self._L.revsim_loss_and_grads(self._h, *[f64p(a) for a in out], f64p(g), f64p(dp)))
        return out[0], out[1], out[2], g, dp

    def rdf(self, term=0, replica=0):
        h = np.zeros(self.terms[term].n_grid)
        self._check(self._L.revsim_rdf(self._h, term, replica, f64p(h)))
        return h

    # --------------------------------------------------------------- drivers
    def _seeds(self, seeds, n_steps):
        s = np.asarray(seeds, dtype=np.uint64)
        if s.ndim == 1:
            s = np.repeat(s[:, None], self.R, axis=1)
        if s.shape != (n_steps, self.R):
            raise ValueError(f"noise seeds must be [n_steps] or [n_steps, n_replicas], got {s.shape}")
        return np.ascontiguousarray(s)

    def _noise(self, noise, n_steps):
        xi = np.ascontiguousarray(noise, dtype=np.float64)
        if xi.size != n_steps * self.n_atoms * 3:
            raise ValueError(f"host noise must hold [n_steps, n_atoms, 3] = "
                             f"[{n_steps}, {self.n_atoms}, 3] values, got {xi.shape}")
        return xi

    def forward(self, seeds, gamma, n_steps, n_steps_loss, dt, calc_loss=True, noise=None):
        """forward_sim from the current state.  ``seeds`` [n_steps] or [n_steps, R] draw the
        Langevin noise on the device; ``noise`` [n_steps, n_atoms, 3] (generate_noise!'s
        output for every step) is used instead when given (seeds may then be None)."""
        loss = np.zeros(self.R)
        if noise is not None:
            xi = self._noise(noise, n_steps)
            self._check(self._L.revsim_forward_noise(self._h, f64p(xi), gamma, n_steps, n_steps_loss,
                                                     dt, 1 if calc_loss else 0, f64p(loss)))
            return loss
        s = self._seeds(seeds, n_steps)
        self._check(self._L.revsim_forward(self._h, u64p(s), gamma, n_steps, n_steps_loss, dt,
                                           1 if calc_loss else 0, f64p(loss)))
        return loss

    def reverse(self, seeds, gamma, n_steps, n_steps_loss, n_steps_trunc, dt, clip=np.inf,
                noise=None):
        """reverse_sim from the forward end state; ``noise`` as for forward (the same array)."""
        loss = np.zeros(self.R)
        g = np.zeros((self.R, self.n_params))
        if noise is not None:
            xi = self._noise(noise, n_steps)
            self._check(self._L.revsim_reverse_noise(self._h, f64p(xi), gamma, n_steps, n_steps_loss,
                                                     n_steps_trunc, dt, clip, f64p(loss), f64p(g)))
            return loss, g
        s = self._seeds(seeds, n_steps)
        self._check(self._L.revsim_reverse(self._h, u64p(s), gamma, n_steps, n_steps_loss,
                                           n_steps_trunc, dt, clip, f64p(loss), f64p(g)))
        return loss, g

    # --------------------------------------------------------- instrumentation
    def set_mlp_precision(self, mode="fp64"):
        """The learned term's network arithmetic: "fp64" (scalar kernels) or "bf16_tc" (tensor
        cores, BF16 operands, FP32 accumulation)."""
        self._check(self._L.revsim_set_mlp_precision(self._h, {"fp64": 0, "bf16_tc": 1}[mode]))

    def mlp_eval(self, r=None):
        """The network on the tensor cores at distances r [3, n] (None: the 1,025 table nodes):
        (u [3, n], du/dr [3, n])."""
        if r is None:
            n, rp = 1025, None
        else:
            r = np.ascontiguousarray(r, dtype=np.float64).reshape(3, -1)
            n, rp = r.shape[1], f64p(r)
        u, du = np.zeros((3, n)), np.zeros((3, n))
        self._check(self._L.revsim_mlp_eval(self._h, n, rp, f64p(u), f64p(du), None))
        return u, du

    def mlp_eval_time(self, r=None):
        """Device milliseconds of one tensor-core evaluation of the network at r [3, n]
        (None: the 1,025 table nodes per type)."""
        ms = ctypes.c_double()
        if r is None:
            self._check(self._L.revsim_mlp_eval(self._h, 1025, None, None, None, ctypes.byref(ms)))
        else:
            r = np.ascontiguousarray(r, dtype=np.float64).reshape(3, -1)
            self._check(self._L.revsim_mlp_eval(self._h, r.shape[1], f64p(r), None, None, ctypes.byref(ms)))
        return ms.value

    def set_pair_mode(self, mode="both_sides"):
        """"both_sides" (each molecule's lanes evaluate its whole row) or "half_shell" (each
        molecule pair evaluated once, the partner's share gathered by a second kernel; mixed
        precision only), revsim_set_pair_mode."""
        code = {"both_sides": 0, "half_shell": 1}[mode]
        self._check(self._L.revsim_set_pair_mode(self._h, code))

    def pair_mode(self):
        """(requested, in effect) pair evaluation modes, revsim_get_pair_mode."""
        req, act = ctypes.c_int32(), ctypes.c_int32()
        self._check(self._L.revsim_get_pair_mode(self._h, ctypes.byref(req), ctypes.byref(act)))
        names = {0: "both_sides", 1: "half_shell"}
        return names[req.value], names[act.value]

    def set_integrator(self, mode="reference"):
        """"reference" (the reference's FP64 step arithmetic) or "exact" (grid increments: with
        gamma = 0 the reverse pass rebuilds the trajectory bit for bit), revsim_set_integrator."""
        self._check(self._L.revsim_set_integrator(self._h, {"reference": 0, "exact": 1}[mode]))

    def set_graph_mode(self, on=True):
        """Capture each forward / reverse pass into a CUDA graph and replay it on later calls
        with the same arguments (revsim_set_graph_mode); the results are the same bits."""
        self._check(self._L.revsim_set_graph_mode(self._h, 1 if on else 0))

    def graph_stats(self):
        """(captures, replays) of the handle's CUDA graphs so far."""
        c, r = ctypes.c_int64(), ctypes.c_int64()
        self._check(self._L.revsim_graph_stats(self._h, ctypes.byref(c), ctypes.byref(r)))
        return c.value, r.value

    def set_kernel_timing(self, on):
        self._check(self._L.revsim_set_kernel_timing(self._h, 1 if on else 0))

    def kernel_time(self, which=0):
        """(total ms, launches) of the reverse (which=0) or forward (1) step kernel."""
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        self._check(self._L.revsim_kernel_time(self._h, which, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def set_launch_shape(self, lanes=0, mols_per_cta=0, unroll=0, which=-1):
        """which: 0 reverse step, 1 forward step, -1 both.  ``lanes`` applies to both
        kernels (forward and reverse forces must be summed in the same order)."""
        self._check(self._L.revsim_set_launch_shape(self._h, which, lanes, mols_per_cta, unroll))

    def launch_shape(self, which=0):
        g, m, u = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._check(self._L.revsim_get_launch_shape(self._h, which, ctypes.byref(g), ctypes.byref(m),
                                                    ctypes.byref(u)))
        return g.value, m.value, u.value

    def autotune(self, dt=0.001):
        """Returns the chosen (lanes, molecules per CTA, unroll) of the reverse and forward kernels."""
        self._check(self._L.revsim_autotune(self._h, dt))
        return self.launch_shape(0), self.launch_shape(1)
