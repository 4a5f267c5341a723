"""The C-ABI library loads and exports every entry point include/ilbm_b200.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

from ilbmrex_b200 import capi

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "ilbm_b200.h").read_text()
    return sorted(set(re.findall(r"\b(ilbm_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(capi.EXPORTS)


def test_library_exports_every_declared_symbol():
    if not capi.LIB_PATH.exists():
        pytest.fail("libilbm_b200.so is not built (python -m ilbmrex_b200.build_lib)")
    lib = ctypes.CDLL(str(capi.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    capi.lib()  # signatures bind


def test_error_path_without_device_state():
    L = capi.lib()
    h = ctypes.c_void_p()
    lat = capi.Lattice_t()
    lat.q = 5  # not a supported lattice
    rc = L.ilbm_create(ctypes.byref(lat), 0, 0, None, ctypes.byref(h))
    assert rc != 0
    assert b"lattice" in L.ilbm_last_error()
