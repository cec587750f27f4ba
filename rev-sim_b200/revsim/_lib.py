"""ctypes binding of librevsim.so (include/revsim.h).

The library is built in-tree by ``rev-sim_b200/build.py``.  There is no CPU
fallback: if the library or a CUDA device is missing, the calls fail loudly.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "librevsim.so")

OK = 0
ERRORS = {
    -1: "REVSIM_ERR_BADARG",
    -2: "REVSIM_ERR_CUDA",
    -3: "REVSIM_ERR_NLIST_OVERFLOW",
    -4: "REVSIM_ERR_NAN",
    -5: "REVSIM_ERR_TIMEOUT",
    -6: "REVSIM_ERR_GEOMETRY",
    -7: "REVSIM_ERR_STATE",
    -8: "REVSIM_ERR_NOMEM",
}

# Every symbol include/revsim.h declares.
EXPORTS = [
    "revsim_create", "revsim_destroy", "revsim_last_error", "revsim_device_status",
    "revsim_sizes", "revsim_set_params", "revsim_set_state", "revsim_get_state",
    "revsim_set_loss", "revsim_neighbor_pairs", "revsim_forces", "revsim_force_vjp",
    "revsim_noise", "revsim_loss_grad", "revsim_rdf", "revsim_forward", "revsim_reverse",
    "revsim_stream", "revsim_launch_count", "revsim_set_kernel_timing", "revsim_kernel_time",
    "revsim_set_launch_shape", "revsim_get_launch_shape", "revsim_autotune",
    "revsim_probe_fp32_tflops", "revsim_rdf_loss_grad_noalloc", "revsim_energy_grad",
    "revsim_set_enth_vap", "revsim_loss_parts", "revsim_loss_and_grads", "revsim_set_barostat",
    "revsim_barostat_state", "revsim_set_box", "revsim_probe_fp64_tflops",
    "revsim_forward_noise", "revsim_reverse_noise", "revsim_set_graph_mode", "revsim_graph_stats",
    "revsim_set_mlp_precision", "revsim_mlp_eval", "revsim_set_integrator",
    "revsim_set_pair_mode", "revsim_get_pair_mode",
]

# Every symbol include/revsim_sw.h declares.
SW_EXPORTS = [
    "revsim_sw_create", "revsim_sw_destroy", "revsim_sw_last_error", "revsim_sw_set_params",
    "revsim_sw_set_state", "revsim_sw_get_state", "revsim_sw_set_loss", "revsim_sw_forces",
    "revsim_sw_force_vjp", "revsim_sw_stress", "revsim_sw_loss_grad", "revsim_sw_noise",
    "revsim_sw_active_pairs", "revsim_sw_forward", "revsim_sw_reverse", "revsim_sw_stream",
    "revsim_sw_launch_count", "revsim_sw_set_kernel_timing", "revsim_sw_kernel_time",
    "revsim_sw_set_lanes",
]


# Every symbol include/revsim_gas.h declares.
GAS_EXPORTS = [
    "revsim_gas_create", "revsim_gas_destroy", "revsim_gas_last_error", "revsim_gas_n_params",
    "revsim_gas_set_params", "revsim_gas_set_state", "revsim_gas_get_state", "revsim_gas_forces",
    "revsim_gas_force_vjp", "revsim_gas_energy", "revsim_gas_forward", "revsim_gas_reverse",
    "revsim_gas_stream", "revsim_gas_launch_count", "revsim_gas_set_kernel_timing",
    "revsim_gas_kernel_time", "revsim_gas_set_rdf",
]


class RevsimError(RuntimeError):
    def __init__(self, code, msg):
        self.code = code
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")


class SystemDesc(ctypes.Structure):
    _fields_ = [
        ("n_replicas", ctypes.c_int32),
        ("n_mol", ctypes.POINTER(ctypes.c_int32)),
        ("box", ctypes.POINTER(ctypes.c_double)),
        ("temp", ctypes.POINTER(ctypes.c_double)),
        ("inter_type", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("m_O", ctypes.c_double),
        ("m_H", ctypes.c_double),
        ("coulomb_const", ctypes.c_double),
        ("crf_const", ctypes.c_double),
        ("cutoff", ctypes.c_double),
        ("nl_cutoff", ctypes.c_double),
        ("kB", ctypes.c_double),
        ("n_steps_nf", ctypes.c_int32),
        ("n_steps_log", ctypes.c_int32),
        ("nl_mode", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("mlp", ctypes.c_int32),
    ]


class BarostatDesc(ctypes.Structure):
    _fields_ = [
        ("pressure", ctypes.c_double),
        ("n_steps", ctypes.c_int32),
        ("scale_factor", ctypes.c_double),
        ("scale_increment", ctypes.c_double),
        ("max_volume_frac", ctypes.c_double),
        ("seed", ctypes.c_uint64),
    ]


class SwDesc(ctypes.Structure):
    _fields_ = [
        ("n_replicas", ctypes.c_int32),
        ("n_atoms", ctypes.POINTER(ctypes.c_int32)),
        ("box", ctypes.POINTER(ctypes.c_double)),
        ("temp", ctypes.POINTER(ctypes.c_double)),
        ("precision", ctypes.c_int32),
        ("mass", ctypes.c_double),
        ("kB", ctypes.c_double),
        ("skin", ctypes.c_double),
        ("n_steps_nf", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("mlp", ctypes.c_int32),
    ]


class GasDesc(ctypes.Structure):
    _fields_ = [
        ("n_water", ctypes.c_int32), ("n_gas", ctypes.c_int32), ("box", ctypes.c_double),
        ("inter_type", ctypes.c_int32), ("temp", ctypes.c_double), ("m_O", ctypes.c_double),
        ("m_H", ctypes.c_double), ("coulomb_const", ctypes.c_double), ("cutoff", ctypes.c_double),
        ("nl_cutoff", ctypes.c_double), ("n_steps_nf", ctypes.c_int32), ("kB", ctypes.c_double),
        ("kb_w", ctypes.c_double), ("r0_w", ctypes.c_double), ("ka_w", ctypes.c_double),
        ("th0_w", ctypes.c_double), ("kb_g", ctypes.c_double), ("r0_g", ctypes.c_double),
        ("n_mol_ev", ctypes.c_int32), ("device", ctypes.c_int32), ("precision", ctypes.c_int32),
    ]


class SwLossC(ctypes.Structure):
    _fields_ = [("weight", ctypes.c_double), ("vel_term", ctypes.c_int32),
                ("target", ctypes.POINTER(ctypes.c_double))]


class RdfTermC(ctypes.Structure):
    _fields_ = [
        ("sel1", ctypes.c_int32), ("sel2", ctypes.c_int32),
        ("x_min", ctypes.c_double), ("step", ctypes.c_double), ("width", ctypes.c_double),
        ("exp_cutoff", ctypes.c_double), ("n_grid", ctypes.c_int32),
        ("slice_start", ctypes.c_int32), ("slice_stride", ctypes.c_int32),
        ("n_target", ctypes.c_int32), ("norm", ctypes.c_int32), ("weight", ctypes.c_double),
    ]


_lib = None


def load(path=LIB_PATH):
    """Load librevsim.so and declare the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RevsimError(-2, f"{path} is missing: build it with rev-sim_b200/build.py")
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    vp, i32, i64, d = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    pd, pi32, pi64, pu64 = P(ctypes.c_double), P(ctypes.c_int32), P(ctypes.c_int64), P(ctypes.c_uint64)
    sig = {
        "revsim_create": (i32, [P(SystemDesc), P(vp)]),
        "revsim_destroy": (None, [vp]),
        "revsim_last_error": (ctypes.c_char_p, [vp]),
        "revsim_device_status": (i32, [vp, pi32]),
        "revsim_sizes": (i32, [vp, pi64, pi32]),
        "revsim_set_params": (i32, [vp, pd, i32]),
        "revsim_set_state": (i32, [vp, pd, pd]),
        "revsim_get_state": (i32, [vp, pd, pd]),
        "revsim_set_loss": (i32, [vp, i32, P(RdfTermC), P(pd)]),
        "revsim_neighbor_pairs": (i32, [vp, i32, pi32, i64, pi64]),
        "revsim_forces": (i32, [vp, pd]),
        "revsim_force_vjp": (i32, [vp, pd, pd, pd, pd, pd]),
        "revsim_noise": (i32, [vp, pu64, pd]),
        "revsim_energy_grad": (i32, [vp, pd, pd]),
        "revsim_loss_grad": (i32, [vp, pd, pd]),
        "revsim_set_enth_vap": (i32, [vp, i32, d, d, d]),
        "revsim_set_barostat": (i32, [vp, P(BarostatDesc)]),
        "revsim_barostat_state": (i32, [vp, pd, pd, pi64, pi64]),
        "revsim_set_box": (i32, [vp, pd]),
        "revsim_loss_parts": (i32, [vp, pd, pd]),
        "revsim_loss_and_grads": (i32, [vp, pd, pd, pd, pd, pd]),
        "revsim_rdf": (i32, [vp, i32, i32, pd]),
        "revsim_forward": (i32, [vp, pu64, d, i32, i32, d, i32, pd]),
        "revsim_reverse": (i32, [vp, pu64, d, i32, i32, i32, d, d, pd, pd]),
        "revsim_forward_noise": (i32, [vp, pd, d, i32, i32, d, i32, pd]),
        "revsim_set_graph_mode": (i32, [vp, i32]),
        "revsim_set_integrator": (i32, [vp, i32]),
        "revsim_set_pair_mode": (i32, [vp, i32]),
        "revsim_get_pair_mode": (i32, [vp, pi32, pi32]),
        "revsim_set_mlp_precision": (i32, [vp, i32]),
        "revsim_mlp_eval": (i32, [vp, i32, pd, pd, pd, pd]),
        "revsim_graph_stats": (i32, [vp, pi64, pi64]),
        "revsim_reverse_noise": (i32, [vp, pd, d, i32, i32, i32, d, d, pd, pd]),
        "revsim_stream": (vp, [vp]),
        "revsim_launch_count": (i64, [vp]),
        "revsim_set_kernel_timing": (i32, [vp, i32]),
        "revsim_kernel_time": (i32, [vp, i32, pd, pi64]),
        "revsim_set_launch_shape": (i32, [vp, i32, i32, i32, i32]),
        "revsim_get_launch_shape": (i32, [vp, i32, pi32, pi32, pi32]),
        "revsim_autotune": (i32, [vp, d]),
        "revsim_probe_fp32_tflops": (i32, [i32, pd]),
        "revsim_probe_fp64_tflops": (i32, [i32, pd]),
        "revsim_rdf_loss_grad_noalloc": (i32, [vp, i32, d, P(RdfTermC), vp, vp, vp, vp]),
        "revsim_sw_create": (i32, [P(SwDesc), P(vp)]),
        "revsim_sw_destroy": (None, [vp]),
        "revsim_sw_last_error": (ctypes.c_char_p, [vp]),
        "revsim_sw_set_params": (i32, [vp, pd, i32]),
        "revsim_sw_set_state": (i32, [vp, pd, pd]),
        "revsim_sw_get_state": (i32, [vp, pd, pd]),
        "revsim_sw_set_loss": (i32, [vp, P(SwLossC)]),
        "revsim_sw_forces": (i32, [vp, pd]),
        "revsim_sw_force_vjp": (i32, [vp, pd, pd, pd, pd, pd]),
        "revsim_sw_stress": (i32, [vp, i32, pd]),
        "revsim_sw_loss_grad": (i32, [vp, pd, pd, pd, pd]),
        "revsim_sw_noise": (i32, [vp, pu64, pd]),
        "revsim_sw_active_pairs": (i32, [vp, pi32, i64, pi64]),
        "revsim_sw_forward": (i32, [vp, pu64, d, i32, i32, i32, d, i32, pd, pi32]),
        "revsim_sw_reverse": (i32, [vp, pu64, d, i32, i32, i32, d, pd, pd]),
        "revsim_sw_stream": (i32, [vp, P(vp)]),
        "revsim_sw_launch_count": (i32, [vp, pi64]),
        "revsim_sw_set_kernel_timing": (i32, [vp, i32]),
        "revsim_sw_kernel_time": (i32, [vp, i32, pd, pi64]),
        "revsim_sw_set_lanes": (i32, [vp, i32]),
        "revsim_gas_create": (i32, [P(GasDesc), P(vp)]),
        "revsim_gas_destroy": (i32, [vp]),
        "revsim_gas_last_error": (ctypes.c_char_p, [vp]),
        "revsim_gas_n_params": (i32, [i32]),
        "revsim_gas_set_params": (i32, [vp, pd, i32]),
        "revsim_gas_set_state": (i32, [vp, pd, pd]),
        "revsim_gas_get_state": (i32, [vp, pd, pd]),
        "revsim_gas_forces": (i32, [vp, pd]),
        "revsim_gas_force_vjp": (i32, [vp, pd, pd, pd, pd, pd]),
        "revsim_gas_energy": (i32, [vp, pd, pd]),
        "revsim_gas_forward": (i32, [vp, pu64, d, i32, i32, d, i32, i32, pd, pd, pd]),
        "revsim_gas_reverse": (i32, [vp, pu64, d, i32, i32, i32, d, i32, pd, pd, pd]),
        "revsim_gas_stream": (vp, [vp]),
        "revsim_gas_launch_count": (i64, [vp]),
        "revsim_gas_set_kernel_timing": (i32, [vp, i32]),
        "revsim_gas_kernel_time": (i32, [vp, i32, pd, pi64]),
        "revsim_gas_set_rdf": (i32, [vp, i32, P(RdfTermC), P(pd)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def f64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def u64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def as_f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a
