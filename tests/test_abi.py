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
    missing = [s for s in declared_symbols() + declared_symbols(SW_HEADER) if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    from revsim import EXPORTS, SW_EXPORTS
    assert sorted(EXPORTS) == declared_symbols()
    assert sorted(SW_EXPORTS) == declared_symbols(SW_HEADER)


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
