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


def test_query_config_validation_without_device():
    """gvx_set_query_config is host-only: shapes outside threads {64,128,256,512}
    x blocks_per_sm [1,64] are refused with GVX_ERR_INVALID_ARG (1), valid ones
    accepted; the library default (256 x 16) is restored at the end."""
    import gvx._abi as abi
    lib = abi.lib()
    for threads, cap, want in [(64, 1, 0), (512, 64, 0), (128, 32, 0), (96, 16, 1), (1024, 16, 1), (256, 0, 1),
                               (256, 65, 1)]:
        c = abi.QueryConfig(threads, cap, 0.0)
        assert lib.gvx_set_query_config(ctypes.byref(c)) == want, (threads, cap)
    assert lib.gvx_set_query_config(None) == 1
    assert lib.gvx_set_query_config(ctypes.byref(abi.QueryConfig(256, 16, 0.0))) == 0
