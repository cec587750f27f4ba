"""ctypes binding of the FP64 CPU oracle (oracle/revsim_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` as the checker.  The product path never imports it.
"""

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc_revsim.so")
_lib = None

_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double
_PD = ctypes.POINTER(ctypes.c_double)
_PI32 = ctypes.POINTER(ctypes.c_int32)
_PU64 = ctypes.POINTER(ctypes.c_uint64)


class OrcSystem(ctypes.Structure):
    _fields_ = [("n_mol", _I32), ("box", _D), ("m_O", _D), ("m_H", _D), ("inter_type", _I32),
                ("coulomb_const", _D), ("crf_const", _D), ("cutoff", _D), ("nl_cutoff", _D),
                ("n_steps_nf", _I32), ("kB", _D), ("temp", _D), ("mlp", _I32)]


class OrcRdfTerm(ctypes.Structure):
    _fields_ = [("sel1", _I32), ("sel2", _I32), ("x_min", _D), ("step", _D), ("width", _D),
                ("exp_cutoff", _D), ("n_grid", _I32), ("slice_start", _I32),
                ("slice_stride", _I32), ("n_target", _I32), ("target", _PD), ("norm", _I32),
                ("weight", _D)]


class OrcLoss(ctypes.Structure):
    _fields_ = [("n_terms", _I32), ("terms", ctypes.POINTER(OrcRdfTerm)), ("enth_vap", _I32),
                ("u_gas", _D), ("rt", _D), ("target", _D)]


class OrcBarostat(ctypes.Structure):
    _fields_ = [("pressure", _D), ("n_steps", _I32), ("volume_scale", _D), ("scale_increment", _D),
                ("max_volume_frac", _D), ("seed", ctypes.c_uint64), ("n_attempted", _I64),
                ("n_accepted", _I64), ("n_draws", _I64), ("n_accepted_total", _I64)]


class OrcGasSystem(ctypes.Structure):
    _fields_ = [("n_water", _I32), ("n_gas", _I32), ("box", _D), ("m_O", _D), ("m_H", _D),
                ("inter_type", _I32), ("coulomb_const", _D), ("crf_const", _D), ("cutoff", _D),
                ("nl_cutoff", _D), ("n_steps_nf", _I32), ("kB", _D), ("temp", _D), ("kb_w", _D),
                ("r0_w", _D), ("ka_w", _D), ("th0_w", _D), ("kb_g", _D), ("r0_g", _D),
                ("n_mol_ev", _I32)]


class OrcSwSystem(ctypes.Structure):
    _fields_ = [("n_atoms", _I32), ("box", _D), ("mass", _D), ("kB", _D), ("temp", _D),
                ("mlp", _I32)]


class OrcSwLoss(ctypes.Structure):
    _fields_ = [("weight", _D), ("target", _D * 9), ("vel_term", _I32)]


def build(force=False):
    """Compile the oracle with its Makefile (gcc, OpenMP, no FMA contraction)."""
    srcs = ["revsim_oracle.c", "revsim_oracle.h", "sw_oracle.c", "sw_oracle.h", "mlp_oracle.c",
            "mlp_oracle.h", "gas_oracle.c", "gas_oracle.h", "Makefile"]
    if force or not os.path.exists(_LIB_PATH) or any(
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, f)) for f in srcs):
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "liborc_revsim.so"],
                       check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_n_params.restype = _I32
        L.orc_neighbor_pairs.restype = _I64
        L.orc_neighbor_pairs.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PI32, _I64]
        L.orc_forces.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PI32, _I64, _PD]
        L.orc_forces_grads.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PI32, _I64, _PD,
                                       _PD, _PD, _PD]
        L.orc_energy.restype = _D
        L.orc_energy.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PI32, _I64]
        L.orc_noise.argtypes = [ctypes.POINTER(OrcSystem), ctypes.c_uint64, _D, _PD]
        L.orc_rdf.argtypes = [ctypes.POINTER(OrcSystem), ctypes.POINTER(OrcRdfTerm), _PD, _PD]
        L.orc_loss_grad.restype = _D
        L.orc_loss_grad.argtypes = [ctypes.POINTER(OrcSystem), ctypes.POINTER(OrcLoss), _PD, _PD]
        L.orc_forward_sim.restype = _D
        L.orc_forward_sim.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PD, _PU64, _D, _I32,
                                      _I32, _D, _I32, ctypes.POINTER(OrcLoss), _I32, _PD, _PD,
                                      _PD]
        L.orc_reverse_sim.restype = _D
        L.orc_reverse_sim.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PD, _PU64, _D, _I32,
                                      _I32, _I32, _D, _I32, _PD, _PD, _D,
                                      ctypes.POINTER(OrcLoss), _PD, _PD]
        L.orc_forward_sim_hn.restype = _D
        L.orc_forward_sim_hn.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PD, _PD, _D, _I32,
                                         _I32, _D, _I32, ctypes.POINTER(OrcLoss), _I32, _PD, _PD, _PD]
        L.orc_reverse_sim_hn.restype = _D
        L.orc_reverse_sim_hn.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PD, _PD, _D, _I32,
                                         _I32, _I32, _D, _I32, _PD, _PD, _D, ctypes.POINTER(OrcLoss),
                                         _PD, _PD]
        L.orc_loss_and_grads.restype = _D
        L.orc_loss_and_grads.argtypes = [ctypes.POINTER(OrcSystem), _PD, ctypes.POINTER(OrcLoss),
                                         _PD, _PD, _PD, _PD]
        L.orc_barostat_uniform.restype = _D
        L.orc_barostat_uniform.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.orc_barostat_attempt.restype = _I32
        L.orc_barostat_attempt.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PI32, _I64,
                                           ctypes.POINTER(OrcBarostat)]
        L.orc_forward_sim_barostat.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PD, _PU64, _D,
                                               _I32, _D, ctypes.POINTER(OrcBarostat)]
        L.orc_num_threads.restype = _I32
        L.orc_set_num_threads.argtypes = [_I32]
        L.orc_energy_grads.restype = _D
        L.orc_energy_grads.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PI32, _I64, _PD]
        L.orc_system_n_params.restype = _I32
        L.orc_system_n_params.argtypes = [ctypes.POINTER(OrcSystem)]
        L.orc_contract.argtypes = [ctypes.POINTER(OrcSystem), _PD, _PD, _PI32, _I64, _PD, _PD]
        L.orc_mlp_nodes.argtypes = [_PD, _D, _PD, _PD]
        L.orc_mlp_table.argtypes = [_PD, _D, _PD]
        L.orc_mlp_pair.argtypes = [_PD, _I32, _D, _D, _PD, _PD, _PD]
        L.orc_mlp_backprop.argtypes = [_PD, _D, _PD, _PD]
        L.orc_mlp_init.argtypes = [ctypes.c_uint64, _PD]
        L.orc_vec1d.restype = _D
        L.orc_vec1d.argtypes = [_D, _D, _D]
        PS, PL = ctypes.POINTER(OrcSwSystem), ctypes.POINTER(OrcSwLoss)
        L.orc_sw_n_params.restype = _I32
        L.orc_sw_n_params.argtypes = [PS]
        L.orc_sw_contract.argtypes = [PS, _PD, _PD, _PD, _PD]
        L.orc_mlp_nodes_n.argtypes = [_PD, _I32, _D, _D, _PD, _PD]
        L.orc_mlp_table_n.argtypes = [_PD, _I32, _D, _D, _PD]
        L.orc_mlp_backprop_n.argtypes = [_PD, _I32, _D, _D, _PD, _PD]
        L.orc_sw_energy.restype = _D
        L.orc_sw_energy.argtypes = [PS, _PD, _PD]
        L.orc_sw_forces.argtypes = [PS, _PD, _PD, _PD]
        L.orc_sw_pairs.restype = _I64
        L.orc_sw_pairs.argtypes = [PS, _PD, _PD, _PI32, _I64]
        L.orc_sw_forces_grads.argtypes = [PS, _PD, _PD, _PD, _PD, _PD, _PD]
        L.orc_sw_stress.argtypes = [PS, _PD, _PD, _PD, _I32, _PD]
        L.orc_sw_loss_grad.restype = _D
        L.orc_sw_loss_grad.argtypes = [PS, _PD, PL, _PD, _PD, _PD, _PD, _PD]
        L.orc_sw_noise.argtypes = [PS, ctypes.c_uint64, _PD]
        L.orc_sw_forward_sim.restype = _D
        L.orc_sw_forward_sim.argtypes = [PS, _PD, _PD, _PD, _PU64, _D, _I32, _I32, _I32, _D, PL,
                                         _I32, _PD, _PD]
        L.orc_sw_reverse_sim.restype = _D
        L.orc_sw_reverse_sim.argtypes = [PS, _PD, _PD, _PD, _PU64, _D, _I32, _I32, _I32, _I32, _D,
                                         _PD, _PD, PL, _PD]
        PG = ctypes.POINTER(OrcGasSystem)
        L.orc_gas_n_params.restype = _I32
        L.orc_gas_n_params.argtypes = [_I32]
        L.orc_gas_neighbor_pairs.restype = _I64
        L.orc_gas_neighbor_pairs.argtypes = [PG, _PD, _PI32, _I64]
        L.orc_gas_forces.argtypes = [PG, _PD, _PD, _PI32, _I64, _PD]
        L.orc_gas_forces_grads.argtypes = [PG, _PD, _PD, _PI32, _I64, _PD, _PD, _PD, _PD, _PD]
        L.orc_gas_energy.restype = _D
        L.orc_gas_energy.argtypes = [PG, _PD, _PD, _PI32, _I64, _PD]
        L.orc_gas_noise.argtypes = [PG, ctypes.c_uint64, _PD]
        L.orc_gas_centres.argtypes = [PG, _PD, _PD]
        L.orc_gas_diffusion_D.restype = _D
        L.orc_gas_diffusion_D.argtypes = [_PD, _I32, _I32, _D, _D, _PD]
        L.orc_gas_loss_final.restype = _D
        L.orc_gas_loss_final.argtypes = [_I32, _PD, _I32, _I32, _D, _D, _D, _D, _PD, _PD]
        L.orc_gas_ev_point.restype = _D
        L.orc_gas_ev_point.argtypes = [PG, _PD, _PD, _I32, _PD, _PD]
        L.orc_gas_forward_sim.restype = _D
        L.orc_gas_forward_sim.argtypes = [PG, _PD, _PD, _PD, _PU64, _D, _I32, _I32, _D, _I32, _I32,
                                          _PD, _PD, _PD, _PD, ctypes.POINTER(OrcLoss)]
        L.orc_gas_reverse_sim.restype = _D
        L.orc_gas_reverse_sim.argtypes = [PG, _PD, _PD, _PD, _PU64, _D, _I32, _I32, _I32, _D, _I32,
                                          _PD, _PD, _PD, _PD, _PD, ctypes.POINTER(OrcLoss)]
        _lib = L
    return _lib


def _pd(a):
    return a.ctypes.data_as(_PD)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


INTER = {"lj": 0, "dexp": 1, "buck": 2, "ljsc": 3, "buff": 4}


def make_system(n_mol, box, inter_type="lj", temp=295.15, *, m_O=15.99943, m_H=1.007947,
                coulomb_const=138.93545764438196, crf_const=None, cutoff=1.0, nl_cutoff=1.2,
                n_steps_nf=20, kB=0.00831446261815324, mlp=False):
    if crf_const is None:
        crf_const = (1.0 / cutoff**3) * ((78.3 - 1) / (2 * 78.3 + 1))
    return OrcSystem(n_mol, box, m_O, m_H, INTER[inter_type], coulomb_const, crf_const, cutoff,
                     nl_cutoff, n_steps_nf, kB, temp, 1 if mlp else 0)


@dataclass
class RdfTerm:
    """One smoothed-RDF loss term (see orc_rdf_term in revsim_oracle.h)."""
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
    _keep: list = field(default_factory=list, repr=False)

    def c(self):
        t = _f64(self.target)
        self._keep = [t]
        return OrcRdfTerm(self.sel1, self.sel2, self.x_min, self.step, self.width,
                          self.exp_cutoff, self.n_grid, self.slice_start, self.slice_stride,
                          len(t), _pd(t), self.norm, self.weight)


# loss_enth_vap constants (water.jl:740-753), kJ/mol
ENTH_U_GAS, ENTH_RT, ENTH_TARGET = 3.69, 2.45, 44.12 + 2.8


class Loss:
    """RDF terms plus, with ``enth_vap``, the enthalpy-of-vaporisation term."""

    def __init__(self, terms, enth_vap=False, u_gas=ENTH_U_GAS, rt=ENTH_RT, target=ENTH_TARGET):
        self.terms = list(terms)
        self._arr = (OrcRdfTerm * max(len(self.terms), 1))(*[t.c() for t in self.terms])
        self.c = OrcLoss(len(self.terms), self._arr, 1 if enth_vap else 0, u_gas, rt, target)


def n_params(s):
    return lib().orc_system_n_params(ctypes.byref(s))


def n_classical_params(s):
    return lib().orc_n_params(s.inter_type)


def neighbor_pairs(s, x):
    x = _f64(x)
    cap = 400 * 3 * s.n_mol + 16
    out = np.zeros((cap, 2), dtype=np.int32)
    n = lib().orc_neighbor_pairs(ctypes.byref(s), _pd(x), out.ctypes.data_as(_PI32), cap)
    if n > cap:
        out = np.zeros((n, 2), dtype=np.int32)
        n = lib().orc_neighbor_pairs(ctypes.byref(s), _pd(x), out.ctypes.data_as(_PI32), n)
    return out[:n].copy()


def forces(s, params, x, pairs):
    x, p = _f64(x), _f64(params)
    pairs = np.ascontiguousarray(pairs, dtype=np.int32)
    F = np.zeros(x.size)
    lib().orc_forces(ctypes.byref(s), _pd(p), _pd(x), pairs.ctypes.data_as(_PI32), len(pairs), _pd(F))
    return F.reshape(-1, 3)


def forces_grads(s, params, x, pairs, w, jac=True):
    """F, the VJP and the Jacobian of the classical parameters."""
    x, p, w = _f64(x), _f64(params), _f64(w)
    pairs = np.ascontiguousarray(pairs, dtype=np.int32)
    P = n_classical_params(s)
    F = np.zeros(x.size)
    G = np.zeros(x.size)
    J = np.zeros(x.size * P) if jac else None
    lib().orc_forces_grads(ctypes.byref(s), _pd(p), _pd(x), pairs.ctypes.data_as(_PI32),
                           len(pairs), _pd(w), _pd(F), _pd(G), _pd(J) if jac else None)
    return F.reshape(-1, 3), G.reshape(-1, 3), (J.reshape(-1, P) if jac else None)


def energy(s, params, x, pairs):
    x, p = _f64(x), _f64(params)
    pairs = np.ascontiguousarray(pairs, dtype=np.int32)
    return lib().orc_energy(ctypes.byref(s), _pd(p), _pd(x), pairs.ctypes.data_as(_PI32), len(pairs))


def energy_grads(s, params, x, pairs):
    """(E, dE/dtheta [P]) at x."""
    x, p = _f64(x), _f64(params)
    pairs = np.ascontiguousarray(pairs, dtype=np.int32)
    g = np.zeros(n_params(s))
    E = lib().orc_energy_grads(ctypes.byref(s), _pd(p), _pd(x), pairs.ctypes.data_as(_PI32),
                               len(pairs), _pd(g))
    return E, g


def noise(s, seed, temp=None):
    xi = np.zeros(9 * s.n_mol)
    lib().orc_noise(ctypes.byref(s), ctypes.c_uint64(int(seed)), s.temp if temp is None else temp,
                    _pd(xi))
    return xi.reshape(-1, 3)


def rdf(s, term, x):
    x = _f64(x)
    h = np.zeros(term.n_grid)
    t = term.c()
    lib().orc_rdf(ctypes.byref(s), ctypes.byref(t), _pd(x), _pd(h))
    return h


def loss_grad(s, loss, x, grad=True):
    x = _f64(x)
    g = np.zeros(x.size) if grad else None
    val = lib().orc_loss_grad(ctypes.byref(s), ctypes.byref(loss.c), _pd(x), _pd(g) if grad else None)
    return val, (g.reshape(-1, 3) if grad else None)


def loss_and_grads(s, params, loss, x):
    """(loss, (l_rdf, l_ev), dL/dx [N, 3], direct dl/dtheta [P]) at x (water.jl:771-786)."""
    x, p = _f64(x), _f64(params)
    parts, g, dp = np.zeros(2), np.zeros(x.size), np.zeros(n_params(s))
    val = lib().orc_loss_and_grads(ctypes.byref(s), _pd(p), ctypes.byref(loss.c), _pd(x),
                                   _pd(parts), _pd(g), _pd(dp))
    return val, (parts[0], parts[1]), g.reshape(-1, 3), dp


def _host_noise(noise, n_steps, n3):
    xi = np.ascontiguousarray(noise, dtype=np.float64)
    if xi.size != n_steps * n3:
        raise ValueError("host noise must hold [n_steps, N, 3] values")
    return xi


def forward_sim(s, params, x, v, seeds, gamma, n_steps, n_steps_loss, dt, loss=None,
                calc_loss=True, n_steps_log=1000, parts=False, noise=None):
    """(x, v, loss, snaps_x, snaps_v), plus (l_rdf, l_ev) when ``parts``.  ``noise``
    [n_steps, N, 3] replaces the seeds' draws (orc_forward_sim_hn)."""
    x, v, p = _f64(x).copy(), _f64(v).copy(), _f64(params)
    n_snap = n_steps // n_steps_log + 1
    sx = np.zeros((n_snap, x.size))
    sv = np.zeros((n_snap, x.size))
    lp = np.zeros(2)
    lc = ctypes.byref(loss.c) if loss is not None else None
    cl = 1 if (calc_loss and loss is not None) else 0
    if noise is not None:
        xi = _host_noise(noise, n_steps, x.size)
        val = lib().orc_forward_sim_hn(ctypes.byref(s), _pd(p), _pd(x), _pd(v), _pd(xi), gamma,
                                       n_steps, n_steps_loss, dt, n_steps_log, lc, cl, _pd(sx),
                                       _pd(sv), _pd(lp))
    else:
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        val = lib().orc_forward_sim(ctypes.byref(s), _pd(p), _pd(x), _pd(v),
                                    seeds.ctypes.data_as(_PU64), gamma, n_steps, n_steps_loss, dt,
                                    n_steps_log, lc, cl, _pd(sx), _pd(sv), _pd(lp))
    out = (x.reshape(-1, 3), v.reshape(-1, 3), val, sx, sv)
    return out + ((lp[0], lp[1]),) if parts else out


def reverse_sim(s, params, x, v, seeds, gamma, n_steps, n_steps_loss, n_steps_trunc, dt,
                snaps_x, snaps_v, loss, clip=float("inf"), n_steps_log=1000, parts=False,
                noise=None):
    """(x0, v0, loss, dl/dtheta), plus (l_rdf, l_ev) when ``parts``; ``noise`` as for
    forward_sim (the same array)."""
    x, v, p = _f64(x).copy(), _f64(v).copy(), _f64(params)
    sx, sv = _f64(snaps_x), _f64(snaps_v)
    g = np.zeros(n_params(s))
    lp = np.zeros(2)
    if noise is not None:
        xi = _host_noise(noise, n_steps, x.size)
        val = lib().orc_reverse_sim_hn(ctypes.byref(s), _pd(p), _pd(x), _pd(v), _pd(xi), gamma,
                                       n_steps, n_steps_loss, n_steps_trunc, dt, n_steps_log,
                                       _pd(sx), _pd(sv), clip, ctypes.byref(loss.c), _pd(g), _pd(lp))
    else:
        seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
        val = lib().orc_reverse_sim(ctypes.byref(s), _pd(p), _pd(x), _pd(v),
                                    seeds.ctypes.data_as(_PU64), gamma, n_steps, n_steps_loss,
                                    n_steps_trunc, dt, n_steps_log, _pd(sx), _pd(sv), clip,
                                    ctypes.byref(loss.c), _pd(g), _pd(lp))
    out = (x.reshape(-1, 3), v.reshape(-1, 3), val, g)
    return out + ((lp[0], lp[1]),) if parts else out


def make_barostat(box, seed, pressure=1.0, n_steps=30, scale_factor=0.01, scale_increment=1.1,
                  max_volume_frac=0.3):
    """MonteCarloBarostatNoUnits(P, T, boundary) with the defaults of water.jl:802-806."""
    return OrcBarostat(pressure, n_steps, box ** 3 * scale_factor, scale_increment, max_volume_frac,
                       int(seed), 0, 0, 0, 0)


def barostat_attempt(s, params, x, pairs, baro):
    """One attempt; returns (accepted, x) with s.box and baro updated in place."""
    x = _f64(x).copy()
    pairs = np.ascontiguousarray(pairs, dtype=np.int32)
    acc = lib().orc_barostat_attempt(ctypes.byref(s), _pd(_f64(params)), _pd(x),
                                     pairs.ctypes.data_as(_PI32), len(pairs), ctypes.byref(baro))
    return bool(acc), x.reshape(-1, 3)


def forward_sim_barostat(s, params, x, v, seeds, gamma, n_steps, dt, baro):
    """Equilibration run with the barostat; returns (x, v); s.box and baro are updated."""
    x, v = _f64(x).copy(), _f64(v).copy()
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    lib().orc_forward_sim_barostat(ctypes.byref(s), _pd(_f64(params)), _pd(x), _pd(v),
                                   seeds.ctypes.data_as(_PU64), gamma, n_steps, dt, ctypes.byref(baro))
    return x.reshape(-1, 3), v.reshape(-1, 3)


def set_threads(n):
    lib().orc_set_num_threads(int(n))


def num_threads():
    return lib().orc_num_threads()


# --------------------------------------------------------------------------------------
# Stillinger-Weber diamond path (sw_oracle.c)

SW_NP = 7


SW_MLP_RC, SW_MLP_WIDTH = 0.25, 0.0125   # the learned radial term (sw_oracle.h)


def make_sw_system(n_atoms, box, temp=298.0, *, mass=12.011, kB=0.00831446261815324, mlp=False):
    return OrcSwSystem(n_atoms, box, mass, kB, temp, 1 if mlp else 0)


def sw_n_params(s):
    return lib().orc_sw_n_params(ctypes.byref(s))


def sw_contract(s, theta, x, acoef):
    """sum_a acoef_a . dF_a/dtheta for every parameter (SW, then the learned term's)."""
    out = np.zeros(sw_n_params(s))
    lib().orc_sw_contract(ctypes.byref(s), _pd(_f64(theta)), _pd(_f64(x)), _pd(_f64(acoef)), _pd(out))
    return out


def make_sw_loss(weight=5e-8, target=None, vel_term=True):
    t = np.zeros(9) if target is None else np.asarray(target, dtype=np.float64).reshape(9)
    return OrcSwLoss(weight, (_D * 9)(*t), 1 if vel_term else 0)


def sw_energy(s, theta, x):
    return lib().orc_sw_energy(ctypes.byref(s), _pd(_f64(theta)), _pd(_f64(x)))


def sw_pairs(s, theta, x):
    """[n, 2] pairs i < j with r / sigma < a, ascending."""
    x = _f64(x)
    cap = 64 * s.n_atoms
    out = np.zeros((cap, 2), dtype=np.int32)
    n = lib().orc_sw_pairs(ctypes.byref(s), _pd(_f64(theta)), _pd(x), out.ctypes.data_as(_PI32), cap)
    return out[:min(n, cap)].copy()


def sw_forces(s, theta, x):
    x = _f64(x)
    F = np.zeros(x.size)
    lib().orc_sw_forces(ctypes.byref(s), _pd(_f64(theta)), _pd(x), _pd(F))
    return F.reshape(-1, 3)


def sw_forces_grads(s, theta, x, w, jac=True):
    x, w = _f64(x), _f64(w)
    F, G = np.zeros(x.size), np.zeros(x.size)
    J = np.zeros(x.size * SW_NP) if jac else None
    lib().orc_sw_forces_grads(ctypes.byref(s), _pd(_f64(theta)), _pd(x), _pd(w), _pd(F), _pd(G),
                              _pd(J) if jac else None)
    return F.reshape(-1, 3), G.reshape(-1, 3), (J.reshape(-1, SW_NP) if jac else None)


def sw_stress(s, theta, x, v, vel_term=True):
    sig = np.zeros(9)
    lib().orc_sw_stress(ctypes.byref(s), _pd(_f64(theta)), _pd(_f64(x)), _pd(_f64(v)),
                        1 if vel_term else 0, _pd(sig))
    return sig.reshape(3, 3)


def sw_loss_grad(s, theta, loss, x, v):
    x, v = _f64(x), _f64(v)
    gx, gv, gp = np.zeros(x.size), np.zeros(x.size), np.zeros(sw_n_params(s))
    val = lib().orc_sw_loss_grad(ctypes.byref(s), _pd(_f64(theta)), ctypes.byref(loss), _pd(x),
                                 _pd(v), _pd(gx), _pd(gv), _pd(gp))
    return val, gx.reshape(-1, 3), gv.reshape(-1, 3), gp


def sw_noise(s, seed):
    xi = np.zeros(3 * s.n_atoms)
    lib().orc_sw_noise(ctypes.byref(s), ctypes.c_uint64(int(seed)), _pd(xi))
    return xi.reshape(-1, 3)


def sw_forward_sim(s, theta, x, v, seeds, gamma, n_steps, n_steps_loss, dt, loss=None,
                   n_steps_buffer=0, calc_loss=True):
    """Forward pass; returns (x, v, loss, snap_x, snap_v) with one snapshot per loss point."""
    x, v = _f64(x).copy(), _f64(v).copy()
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    n_pts = sum(1 for k in range(1, n_steps + 1)
                if (n_steps - k) % n_steps_loss == 0 and k >= n_steps_buffer)
    sx = np.zeros((max(n_pts, 1), x.size))
    sv = np.zeros((max(n_pts, 1), x.size))
    val = lib().orc_sw_forward_sim(ctypes.byref(s), _pd(_f64(theta)), _pd(x), _pd(v),
                                   seeds.ctypes.data_as(_PU64), gamma, n_steps, n_steps_loss,
                                   n_steps_buffer, dt,
                                   ctypes.byref(loss) if loss is not None else None,
                                   1 if (calc_loss and loss is not None) else 0, _pd(sx), _pd(sv))
    return x.reshape(-1, 3), v.reshape(-1, 3), val, sx[:n_pts], sv[:n_pts]


def sw_reverse_sim(s, theta, x, v, seeds, gamma, n_steps, n_steps_loss, n_steps_trunc, dt,
                   snaps_x, snaps_v, loss):
    """Reverse pass over the forward pass's loss points; returns (x, v, loss, dL/dtheta)."""
    x, v = _f64(x).copy(), _f64(v).copy()
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    sx, sv = _f64(snaps_x), _f64(snaps_v)
    g = np.zeros(sw_n_params(s))
    val = lib().orc_sw_reverse_sim(ctypes.byref(s), _pd(_f64(theta)), _pd(x), _pd(v),
                                   seeds.ctypes.data_as(_PU64), gamma, n_steps, n_steps_loss,
                                   n_steps_trunc, len(sx), dt, _pd(sx), _pd(sv),
                                   ctypes.byref(loss), _pd(g))
    return x.reshape(-1, 3), v.reshape(-1, 3), val, g


# --------------------------------------------------------------------------------------
# Learned pair correction (mlp_oracle.c)

MLP_NG, MLP_NT, MLP_H, MLP_NRBF = 1024, 3, 64, 16
MLP_PER_TYPE = MLP_H * MLP_NRBF + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1
MLP_NPARAMS = MLP_NT * MLP_PER_TYPE


def contract(s, params, x, pairs, acoef):
    """sum_a acoef_a . dF_a/dtheta for every parameter (classical, then MLP)."""
    x, p, a = _f64(x), _f64(params), _f64(acoef)
    pairs = np.ascontiguousarray(pairs, dtype=np.int32)
    out = np.zeros(n_params(s))
    lib().orc_contract(ctypes.byref(s), _pd(p), _pd(x), pairs.ctypes.data_as(_PI32), len(pairs),
                       _pd(a), _pd(out))
    return out


def mlp_init(seed=3):
    th = np.zeros(MLP_NPARAMS)
    lib().orc_mlp_init(ctypes.c_uint64(seed), _pd(th))
    return th


def mlp_nodes(theta, rc=1.0):
    u = np.zeros((MLP_NT, MLP_NG + 1))
    du = np.zeros((MLP_NT, MLP_NG + 1))
    lib().orc_mlp_nodes(_pd(_f64(theta)), rc, _pd(u), _pd(du))
    return u, du


def mlp_table(theta, rc=1.0):
    c = np.zeros((MLP_NT, MLP_NG, 4))
    lib().orc_mlp_table(_pd(_f64(theta)), rc, _pd(c))
    return c


def mlp_pair(coef, t, r, rc=1.0):
    u, F, dF = _D(), _D(), _D()
    lib().orc_mlp_pair(_pd(_f64(coef)), t, rc, r, ctypes.byref(u), ctypes.byref(F), ctypes.byref(dF))
    return u.value, F.value, dF.value


def mlp_backprop(theta, coef_adj, rc=1.0):
    out = np.zeros(MLP_NPARAMS)
    lib().orc_mlp_backprop(_pd(_f64(theta)), rc, _pd(_f64(coef_adj)), _pd(out))
    return out


def mlp_table_n(theta, nt, rc, width):
    c = np.zeros((nt, MLP_NG, 4))
    lib().orc_mlp_table_n(_pd(_f64(theta)), nt, rc, width, _pd(c))
    return c


# ------------------------------------------------------------------ gas in water
# diffusion.jl: O2 bond k = 1640.4 kcal/mol/A^2 in kJ/mol/nm^2 and r0 (:46, :1113-1116)
GAS_KB, GAS_R0 = 1640.4 * 4.184 * 100, 0.12074
GAS_LOSS = {"diff": 1, "rdf": 2, "ev": 4, "diff_rdf": 3, "diff_ev": 5, "rdf_ev": 6, "diff_rdf_ev": 7}


def make_gas_system(n_water, n_gas, box, inter_type="lj", temp=295.15, *, m_O=15.99943,
                    m_H=1.007947, coulomb_const=138.93545764438196, cutoff=1.0, nl_cutoff=1.2,
                    n_steps_nf=20, kB=0.00831446261815324, kb_w=462750.4, r0_w=0.09572,
                    ka_w=836.8, th0_w=1.82421813418, kb_g=GAS_KB, r0_g=GAS_R0, n_mol_ev=None):
    crf = (1.0 / cutoff**3) * ((78.3 - 1) / (2 * 78.3 + 1))
    return OrcGasSystem(n_water, n_gas, box, m_O, m_H, INTER[inter_type], coulomb_const, crf,
                        cutoff, nl_cutoff, n_steps_nf, kB, temp, kb_w, r0_w, ka_w, th0_w, kb_g,
                        r0_g, n_water + n_gas if n_mol_ev is None else n_mol_ev)


def gas_n_atoms(s):
    return 3 * s.n_water + 2 * s.n_gas


def gas_n_params(inter_type):
    return lib().orc_gas_n_params(INTER[inter_type] if isinstance(inter_type, str) else inter_type)


def gas_neighbor_pairs(s, x):
    x = _f64(x)
    n = lib().orc_gas_neighbor_pairs(ctypes.byref(s), _pd(x), None, 0)
    pairs = np.zeros((max(n, 1), 2), dtype=np.int32)
    lib().orc_gas_neighbor_pairs(ctypes.byref(s), _pd(x), pairs.ctypes.data_as(_PI32), n)
    return pairs[:n]


def gas_forces(s, p, x, pairs=None):
    x = _f64(x)
    pairs = gas_neighbor_pairs(s, x) if pairs is None else np.ascontiguousarray(pairs, np.int32)
    F = np.zeros(3 * gas_n_atoms(s))
    lib().orc_gas_forces(ctypes.byref(s), _pd(_f64(p)), _pd(x), pairs.ctypes.data_as(_PI32),
                         len(pairs), _pd(F))
    return F.reshape(-1, 3)


def gas_forces_grads(s, p, x, w, acoef, pairs=None):
    """(F, dl_dfi, dl_dp) of calc_F_and_grads! against dl_dfi_prev = w with the contraction
    against acoef."""
    x = _f64(x)
    pairs = gas_neighbor_pairs(s, x) if pairs is None else np.ascontiguousarray(pairs, np.int32)
    n3 = 3 * gas_n_atoms(s)
    F, G = np.zeros(n3), np.zeros(n3)
    dp = np.zeros(gas_n_params(s.inter_type))
    lib().orc_gas_forces_grads(ctypes.byref(s), _pd(_f64(p)), _pd(x), pairs.ctypes.data_as(_PI32),
                               len(pairs), _pd(_f64(w)), _pd(_f64(acoef)), _pd(F), _pd(G), _pd(dp))
    return F.reshape(-1, 3), G.reshape(-1, 3), dp


def gas_energy(s, p, x, pairs=None, grads=False):
    x = _f64(x)
    pairs = gas_neighbor_pairs(s, x) if pairs is None else np.ascontiguousarray(pairs, np.int32)
    dp = np.zeros(gas_n_params(s.inter_type)) if grads else None
    E = lib().orc_gas_energy(ctypes.byref(s), _pd(_f64(p)), _pd(x), pairs.ctypes.data_as(_PI32),
                             len(pairs), _pd(dp) if grads else None)
    return (E, dp) if grads else E


def gas_noise(s, seed):
    xi = np.zeros(3 * gas_n_atoms(s))
    lib().orc_gas_noise(ctypes.byref(s), ctypes.c_uint64(int(seed)), _pd(xi))
    return xi.reshape(-1, 3)


def gas_centres(s, x):
    c = np.zeros(3 * s.n_gas)
    lib().orc_gas_centres(ctypes.byref(s), _pd(_f64(x)), _pd(c))
    return c.reshape(-1, 3)


def gas_diffusion_D(gc, box, loss_frequency, grads=False):
    gc = _f64(gc)
    n_frames, n_gas = gc.shape[0], gc.shape[1]
    g = np.zeros_like(gc) if grads else None
    D = lib().orc_gas_diffusion_D(_pd(gc), n_frames, n_gas, box, loss_frequency,
                                  _pd(g) if grads else None)
    return (D, g) if grads else D


def gas_loss_final(loss_type, gc, box, loss_frequency, ev_sum=0.0, rdf_sum=0.0):
    """(loss, [D m^2/s, l_diff, l_rdf, l_ev], dl_diff/dgc)."""
    gc = _f64(gc)
    out = np.zeros(4)
    g = np.zeros_like(gc)
    l = lib().orc_gas_loss_final(GAS_LOSS[loss_type], _pd(gc), gc.shape[0], gc.shape[1], box,
                                 loss_frequency, ev_sum, rdf_sum, _pd(out), _pd(g))
    return l, out, g


def gas_ev_point(s, p, x, n_blocks):
    """(l, dl/dx, direct dl/dtheta) of one loss point's enthalpy term."""
    g = np.zeros(3 * gas_n_atoms(s))
    dp = np.zeros(gas_n_params(s.inter_type))
    l = lib().orc_gas_ev_point(ctypes.byref(s), _pd(_f64(p)), _pd(_f64(x)), n_blocks, _pd(g), _pd(dp))
    return l, g.reshape(-1, 3), dp


def gas_forward_sim(s, p, x, v, seeds, gamma, n_steps, n_steps_loss, dt, loss_type="diff",
                    calc_loss=True, rdf=None):
    """(x, v, loss, snaps_x, snaps_v, centres, [D, l_diff, l_rdf, l_ev]); rdf: a Loss of RDF
    terms for the rdf loss types."""
    x, v = _f64(x).copy(), _f64(v).copy()
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    n_blocks = 1 if n_steps == 0 else n_steps // n_steps_loss
    n3 = 3 * gas_n_atoms(s)
    sx, sv = np.zeros((n_blocks + 1, n3)), np.zeros((n_blocks + 1, n3))
    gc = np.zeros((n_blocks, s.n_gas, 3))
    out = np.zeros(4)
    l = lib().orc_gas_forward_sim(ctypes.byref(s), _pd(_f64(p)), _pd(x), _pd(v),
                                  seeds.ctypes.data_as(_PU64), gamma, n_steps, n_steps_loss, dt,
                                  GAS_LOSS[loss_type], 1 if calc_loss else 0, _pd(sx), _pd(sv),
                                  _pd(gc), _pd(out), ctypes.byref(rdf.c) if rdf is not None else None)
    return x, v, l, sx, sv, gc, out


def gas_reverse_sim(s, p, x, v, seeds, gamma, n_steps, n_steps_loss, n_steps_trunc, dt, snaps_x,
                    snaps_v, centres, loss_type="diff", rdf=None):
    """(x, v, loss, dl_dp, [D, l_diff, l_rdf, l_ev])."""
    x, v = _f64(x).copy(), _f64(v).copy()
    seeds = np.ascontiguousarray(seeds, dtype=np.uint64)
    dp = np.zeros(gas_n_params(s.inter_type))
    out = np.zeros(4)
    l = lib().orc_gas_reverse_sim(ctypes.byref(s), _pd(_f64(p)), _pd(x), _pd(v),
                                  seeds.ctypes.data_as(_PU64), gamma, n_steps, n_steps_loss,
                                  n_steps_trunc, dt, GAS_LOSS[loss_type], _pd(_f64(snaps_x)),
                                  _pd(_f64(snaps_v)), _pd(_f64(centres)), _pd(dp), _pd(out),
                                  ctypes.byref(rdf.c) if rdf is not None else None)
    return x, v, l, dp, out
