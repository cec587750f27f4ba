"""The C-ABI library: it loads and exports every entry point include/revsim.h declares.
No compute calls (this runs without a GPU)."""

import ctypes
import sys
import os
import re

import pytest

from conftest import PKG, ROOT

HEADER = os.path.join(ROOT, "include", "revsim.h")
SW_HEADER = os.path.join(ROOT, "include", "revsim_sw.h")
GAS_HEADER = os.path.join(ROOT, "include", "revsim_gas.h")


def declared_symbols(header=HEADER):
    src = open(header).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(revsim_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    sys.path.insert(0, PKG)
    import build as b  # rev-sim_b200/build.py
    path = b.build()
    return ctypes.CDLL(path)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "revsim_reverse" in syms and "revsim_forward" in syms
    assert len(syms) >= 20


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() + declared_symbols(SW_HEADER) + declared_symbols(GAS_HEADER)
               if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    from revsim import EXPORTS, GAS_EXPORTS, SW_EXPORTS
    assert sorted(EXPORTS) == declared_symbols()
    assert sorted(SW_EXPORTS) == declared_symbols(SW_HEADER)
    assert sorted(GAS_EXPORTS) == declared_symbols(GAS_HEADER)


def test_error_paths_without_device(lib):
    # Argument validation happens before any CUDA call.
    from revsim import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.revsim_create(None, ctypes.byref(h)) == -1
    assert L.revsim_set_params(None, None, 0) == -1
    assert L.revsim_forward(None, None, 0.0, 0, 0, 0.0, 0, None) == -1
    assert L.revsim_last_error(None) == b"null handle"


def test_sw_error_paths_without_device(lib):
    from revsim import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.revsim_sw_create(None, ctypes.byref(h)) == -1
    assert L.revsim_sw_set_params(None, None, 0) == -1
    assert L.revsim_sw_forward(None, None, 0.0, 0, 1, 0, 0.0, 0, None, None) == -1
    assert L.revsim_sw_last_error(None) == b"null handle"


def test_new_entry_points_reject_a_null_handle(lib):
    from revsim import _lib
    L = _lib.load()
    d = _lib.BarostatDesc(1.0, 30, 0.01, 1.1, 0.3, 0)
    assert L.revsim_set_enth_vap(None, 1, 3.69, 2.45, 46.92) == -1
    assert L.revsim_loss_parts(None, None, None) == -1
    assert L.revsim_loss_and_grads(None, None, None, None, None, None) == -1
    assert L.revsim_set_barostat(None, ctypes.byref(d)) == -1
    assert L.revsim_barostat_state(None, None, None, None, None) == -1
    assert L.revsim_set_box(None, None) == -1
    assert L.revsim_forward_noise(None, None, 0.0, 0, 0, 0.0, 0, None) == -1
    assert L.revsim_reverse_noise(None, None, 0.0, 1, 1, 1, 0.001, 1.0, None, None) == -1


def test_descriptor_validation_before_any_device_call(lib):
    """Invalid descriptions return REVSIM_ERR_BADARG before the library touches CUDA."""
    import numpy as np
    from revsim import _lib, constants as C
    L = _lib.load()
    h = ctypes.c_void_p()
    n = np.array([0], dtype=np.int32)            # a replica without molecules
    box, temp = np.array([3.0]), np.array([295.0])
    pd = ctypes.POINTER(ctypes.c_double)
    desc = _lib.SystemDesc(1, n.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), box.ctypes.data_as(pd),
                           temp.ctypes.data_as(pd), 0, 0, C.O_MASS, C.H_MASS, C.COULOMB_CONST,
                           C.CRF_CONST, 1.0, 1.2, C.KB, 20, 1000, 0, 0, 0)
    assert L.revsim_create(ctypes.byref(desc), ctypes.byref(h)) == -1
    n[0] = 10
    box[0] = 2.3                                  # below twice the 1.2 nm list cutoff
    assert L.revsim_create(ctypes.byref(desc), ctypes.byref(h)) == -1
    box[0] = 3.0
    desc.mlp = 1
    desc.inter_type = 2                           # the learned term needs REVSIM_LJ
    assert L.revsim_create(ctypes.byref(desc), ctypes.byref(h)) == -1


def test_gas_entry_points_without_device(lib):
    """Argument checks of the gas-in-water ABI happen before any CUDA call."""
    from revsim import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.revsim_gas_create(None, ctypes.byref(h)) == -1
    d = _lib.GasDesc()
    d.n_water, d.n_gas, d.box, d.inter_type = 10, 2, 2.0, 0    # box < 2 x 1.2 nm
    assert L.revsim_gas_create(ctypes.byref(d), ctypes.byref(h)) == -6 and not h.value
    d.box, d.inter_type = 3.0, 9
    assert L.revsim_gas_create(ctypes.byref(d), ctypes.byref(h)) == -1
    d.inter_type, d.n_water, d.n_gas = 0, 0, 0
    assert L.revsim_gas_create(ctypes.byref(d), ctypes.byref(h)) == -1
    assert [L.revsim_gas_n_params(t) for t in range(5)] == [5, 7, 7, 7, 7]
    assert L.revsim_gas_n_params(5) == -1
    assert L.revsim_gas_set_params(None, None, 0) == -1
    assert L.revsim_gas_forward(None, None, 0.0, 0, 1, 0.001, 1, 1, None, None, None) == -1
    assert L.revsim_gas_reverse(None, None, 0.0, 0, 1, 1, 0.001, 1, None, None, None) == -1
    assert L.revsim_gas_last_error(None) == b"null handle"
    assert L.revsim_gas_destroy(None) == 0
