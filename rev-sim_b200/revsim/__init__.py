"""revsim: B200 (sm_100a) engine for the reversible-simulation gradient of
greener-group/rev-sim's flexible-water model.

The compute runs in librevsim.so (CUDA, C ABI in include/revsim.h); this package
is the host side: a ctypes binding (``Engine``), the reference's
``forward_sim`` / ``reverse_sim`` signatures (``water``), loss builders (``loss``)
and seeded system generators (``systems``); the Stillinger-Weber diamond engine
(``SwEngine``, C ABI in include/revsim_sw.h) with the diamond entry points in ``sw``; the
gas-in-water engine of diffusion.jl (``gas.GasEngine``, C ABI in include/revsim_gas.h).
"""

from . import constants, diamond, systems
from . import gas
from ._lib import EXPORTS, GAS_EXPORTS, LIB_PATH, SW_EXPORTS, RevsimError, load
from .engine import Engine, RdfTerm
from .loss import oo_l2_term, read_rdf_data, reference_rdf_terms
from .sw import SwEngine
from .water import SimSystem, forward_sim, reverse_sim, reweighting_sim

__all__ = [
    "Engine", "RdfTerm", "RevsimError", "SimSystem", "forward_sim", "reverse_sim",
    "reweighting_sim", "load",
    "constants", "systems", "oo_l2_term", "reference_rdf_terms", "read_rdf_data", "EXPORTS",
    "LIB_PATH", "SW_EXPORTS", "SwEngine", "diamond", "gas", "GAS_EXPORTS",
]
