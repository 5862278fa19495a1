"""The C-ABI library loads without a GPU and exports exactly what
include/gvx.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"GVX_API\s+[\w\s\*]+?\b(gvx_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = _declared("gvx.h")
    assert "gvx_dvm_edt" in names and "gvx_bvm_collide" in names and len(names) >= 30


def test_library_exports_every_declared_symbol():
    import gvx._abi as abi
    lib = abi.lib()
    missing = [n for n in _declared("gvx.h") if not hasattr(lib, n)]
    assert not missing, missing
    # the Python prototypes cover the whole header
    assert set(_declared("gvx.h")) == set(abi.PROTOTYPES)


def test_error_path_without_device():
    import gvx._abi as abi
    lib = abi.lib()
    out = ctypes.c_void_p()
    d = abi.Dims(0, 10, 10)
    st = lib.gvx_dvm_create(ctypes.byref(d), 1.0, ctypes.byref(out))
    assert st == 2 and out.value is None  # GVX_ERR_OUT_OF_DOMAIN before any CUDA call
    assert b"1023" in lib.gvx_last_error()
    d = abi.Dims(10, 10, 1024)
    assert lib.gvx_dvm_create(ctypes.byref(d), 1.0, ctypes.byref(out)) == 2
    with pytest.raises(abi.GvxError):
        abi.call("gvx_dvm_edt", None, 1, 1, 1, None)
