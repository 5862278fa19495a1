"""The allocation-free EDT entry point, gvx_dvm_edt_static_workspace.

It exists for callers that may not allocate device memory once running (a
real-time control loop, a plugin inside a host application that owns all
device memory): it runs the EDT in place on the caller's voxel buffer with a
workspace built into the library.  This test drives it through the C ABI with
ctypes and checks, on three calls in a row, that it returns exactly what the
regular entry point (gvx_dvm_create + gvx_dvm_edt) returns -- the EDT is
integer work, so the tolerance is bit equality, as in the other EDT tests.
The 256^3 map runs first and a small map twice after it, so the small map's
calls meet the counters, stacks and occupancy words a larger map left in the
shared workspace.  After every call the handle-free check must report that
no bounded wait gave up.  This file is collected last so a failure here
comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _regular_edt(abi, dims, side, pts):
    """EDT through the regular entry points; returns (map before, map after)."""
    lib = abi.lib()
    d = abi.Dims(*dims)
    h = ctypes.c_void_p()
    abi.check(lib.gvx_dvm_create(ctypes.byref(d), side, ctypes.byref(h)))
    try:
        p = torch.as_tensor(pts).cuda().contiguous()
        abi.check(lib.gvx_dvm_insert_points(h, ctypes.c_void_p(p.data_ptr()), p.shape[0], None, None))
        ptr = ctypes.c_void_p()
        abi.check(lib.gvx_dvm_info(h, None, None, ctypes.byref(ptr)))
        n = int(np.prod(dims))
        before = torch.empty(n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        _copy_from(ptr.value, before)
        abi.check(lib.gvx_dvm_edt(h, 1, 1, 1, None))
        torch.cuda.synchronize()
        after = torch.empty(n, dtype=torch.int32, device="cuda")
        _copy_from(ptr.value, after)
        return before, after
    finally:
        lib.gvx_dvm_destroy(h)


def _copy_from(device_ptr, dst):
    class _View:
        __cuda_array_interface__ = {"shape": (dst.numel(),), "typestr": "<i4", "data": (device_ptr, False), "version": 3}

    dst.copy_(torch.as_tensor(_View(), device="cuda"))
    torch.cuda.synchronize()


def test_static_workspace_edt_matches_regular_entry_point_twice():
    import gvx._abi as abi
    import workloads

    lib = abi.lib()
    rng = np.random.default_rng(2024)
    sc = workloads.c3_scene()  # 256^3: the largest cube the built-in workspace takes
    small = ((96, 64, 80), 1.0, (rng.random((3000, 3)) * [96, 64, 80]).astype(np.float32))
    cases = [(sc.dims, sc.side, sc.points), small, small]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for dims, side, pts in cases:  # calls in a row on one shared workspace
        before, want = _regular_edt(abi, dims, side, pts)
        buf = before.clone()
        d = abi.Dims(*dims)
        abi.check(lib.gvx_dvm_edt_static_workspace(ctypes.c_void_p(buf.data_ptr()), ctypes.byref(d), stream))
        flags = ctypes.c_uint32(7)
        abi.check(lib.gvx_dvm_edt_static_workspace_check(ctypes.byref(d), ctypes.byref(flags)))
        assert flags.value == 0
        torch.cuda.synchronize()
        assert torch.equal(buf, want), f"static-workspace EDT differs from gvx_dvm_edt on {dims}"


def test_static_workspace_rejects_maps_beyond_its_limit():
    import gvx._abi as abi

    lib = abi.lib()
    dims = abi.Dims(257, 256, 256)  # x rounds up to 288: over the built-in workspace
    buf = torch.full((257 * 256 * 256,), 0x3FFFFFFF, dtype=torch.int32, device="cuda")
    st = lib.gvx_dvm_edt_static_workspace(ctypes.c_void_p(buf.data_ptr()), ctypes.byref(dims), None)
    assert st == 2  # GVX_ERR_OUT_OF_DOMAIN
    assert b"static EDT workspace" in lib.gvx_last_error()
    torch.cuda.synchronize()
    assert bool((buf == 0x3FFFFFFF).all())
