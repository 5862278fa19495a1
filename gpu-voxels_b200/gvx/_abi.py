"""ctypes binding of the C ABI declared in include/gvx.h (lib/libgvx.so).

The library is the product; this module only declares prototypes and turns
a non-zero gvx_status into a GvxError carrying gvx_last_error().  Loading
fails loudly when the built library is missing -- there is no fallback.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libgvx.so")

GVX_OK = 0
STATUS_NAMES = {
    0: "GVX_OK",
    1: "GVX_ERR_INVALID_ARG",
    2: "GVX_ERR_OUT_OF_DOMAIN",
    3: "GVX_ERR_OOM",
    4: "GVX_ERR_CUDA",
    5: "GVX_ERR_TIMEOUT",
    6: "GVX_ERR_NO_DEVICE",
}

GVX_MAX_JOINTS = 16
GVX_MAX_SPHERES = 256


class GvxError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class EdtConfig(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint32), ("fused", ctypes.c_uint32), ("ms", ctypes.c_float)]


class QueryConfig(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_uint32), ("blocks_per_sm", ctypes.c_uint32), ("ms", ctypes.c_float)]


class Dims(ctypes.Structure):
    _fields_ = [("x", ctypes.c_uint32), ("y", ctypes.c_uint32), ("z", ctypes.c_uint32)]


class Arm(ctypes.Structure):
    _fields_ = [
        ("n_joints", ctypes.c_int32),
        ("n_spheres", ctypes.c_int32),
        ("base", ctypes.c_float * 16),
        ("theta", ctypes.c_float * GVX_MAX_JOINTS),
        ("d", ctypes.c_float * GVX_MAX_JOINTS),
        ("a", ctypes.c_float * GVX_MAX_JOINTS),
        ("alpha", ctypes.c_float * GVX_MAX_JOINTS),
        ("link", ctypes.c_int32 * GVX_MAX_SPHERES),
        ("t", ctypes.c_float * GVX_MAX_SPHERES),
        ("r", ctypes.c_float * GVX_MAX_SPHERES),
    ]


_vp = ctypes.c_void_p
_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32
_i32p = ctypes.POINTER(ctypes.c_int32)
_f = ctypes.c_float
_st = ctypes.c_int

# name -> argtypes (all return gvx_status unless listed in _RESTYPES)
PROTOTYPES = {
    "gvx_last_error": [],
    "gvx_version": [],
    "gvx_init_device": [ctypes.c_int],
    "gvx_dvm_create": [ctypes.POINTER(Dims), _f, ctypes.POINTER(_vp)],
    "gvx_dvm_wrap": [ctypes.POINTER(Dims), _f, _vp, ctypes.POINTER(_vp)],
    "gvx_dvm_destroy": [_vp],
    "gvx_dvm_info": [_vp, ctypes.POINTER(Dims), ctypes.POINTER(_f), ctypes.POINTER(_vp)],
    "gvx_dvm_clear": [_vp, _vp],
    "gvx_dvm_insert_points": [_vp, _vp, _u64, _vp, _vp],
    "gvx_dvm_edt": [_vp, _u32, _u32, _u32, _vp],
    "gvx_dvm_edt_pass": [_vp, ctypes.c_int, _vp],
    "gvx_dvm_edt_check": [_vp, ctypes.POINTER(_u32)],
    "gvx_check_bisector_quotient": [ctypes.POINTER(_u64)],
    "gvx_dvm_voxelize_edt": [_vp, _vp, _u64, _vp, _vp],
    "gvx_dvm_autotune": [_vp, ctypes.c_int, ctypes.POINTER(EdtConfig), _vp],
    "gvx_dvm_set_edt_config": [_vp, ctypes.POINTER(EdtConfig)],
    "gvx_dvm_edt_static_workspace": [_vp, ctypes.POINTER(Dims), _vp],
    "gvx_dvm_edt_static_workspace_check": [ctypes.POINTER(Dims), ctypes.POINTER(_u32)],
    "gvx_dvm_sqdist": [_vp, _vp, _u64, _vp, _vp],
    "gvx_dvm_dist": [_vp, _vp, _u64, _vp, _vp],
    "gvx_dvm_gather": [_vp, _vp, _u64, _vp, _vp],
    "gvx_dvm_sqdist_map": [_vp, _vp, _vp],
    "gvx_query_trilinear": [_vp, _vp, _u64, _vp, _vp, _vp],
    "gvx_query_trilinear_bwd": [_vp, _vp, _u64, _vp, _vp, _vp],
    "gvx_query_autotune": [_vp, _vp, _u64, _vp, _vp, ctypes.c_int, ctypes.POINTER(QueryConfig), _vp],
    "gvx_set_query_config": [ctypes.POINTER(QueryConfig)],
    "gvx_sphere_clearance": [_vp, ctypes.POINTER(Arm), _vp, _u64, _vp, _vp],
    "gvx_traj_cost": [_vp, ctypes.POINTER(Arm), _vp, _u64, _u32, _f, _vp, _vp],
    "gvx_traj_cost_bwd": [_vp, ctypes.POINTER(Arm), _vp, _u64, _u32, _f, _vp, _vp, _vp],
    "gvx_batch_create": [ctypes.POINTER(_vp), _u32, ctypes.POINTER(_vp)],
    "gvx_batch_destroy": [_vp],
    "gvx_batch_clear": [_vp, _vp],
    "gvx_batch_insert_points": [_vp, _vp, _vp, _u64, _vp],
    "gvx_batch_edt": [_vp, _vp],
    "gvx_batch_edt_check": [_vp, ctypes.POINTER(_u32)],
    "gvx_batch_voxelize_edt": [_vp, _vp, _vp, _u64, _vp],
    "gvx_batch_autotune": [_vp, ctypes.c_int, ctypes.POINTER(EdtConfig), _vp],
    "gvx_batch_query_trilinear": [_vp, _vp, _vp, _u64, _vp, _vp, _vp],
    "gvx_batch_graph_capture": [_vp, _vp, _vp, _u64, _vp, _vp, _u64, _vp, _vp, _vp],
    "gvx_batch_graph_launch": [_vp, _vp],
    "gvx_bvm_create": [ctypes.POINTER(Dims), _f, ctypes.POINTER(_vp)],
    "gvx_bvm_destroy": [_vp],
    "gvx_bvm_info": [_vp, ctypes.POINTER(Dims), ctypes.POINTER(_f), ctypes.POINTER(_vp)],
    "gvx_bvm_clear": [_vp, _vp],
    "gvx_bvm_insert_points": [_vp, _vp, _u64, _u32, _vp, _vp],
    "gvx_bvm_clear_bits": [_vp, _vp, _vp],
    "gvx_bvm_collide_pvm": [_vp, _vp, _f, _vp, ctypes.c_int, _vp, _vp],
    "gvx_blist_collide_pvm": [_vp, _vp, _f, _vp, ctypes.c_int, _vp, _vp],
    "gvx_blist_clear_bits": [_vp, _vp, _vp],
    "gvx_blist_shift_swept_volume_ids": [_vp, _u32, _vp],
    "gvx_bvm_shift_swept_volume_ids": [_vp, _u32, _vp],
    "gvx_bvm_insert_meta_points_self_coll": [_vp, _vp, ctypes.POINTER(_u64), _u32, _vp, _vp, _vp,
                                             ctypes.POINTER(ctypes.c_int), _vp, _vp],
    "gvx_bvm_collide": [_vp, _vp, _i32p, ctypes.c_int, _vp, _vp],
    "gvx_pvm_create": [ctypes.POINTER(Dims), _f, ctypes.POINTER(_vp)],
    "gvx_pvm_destroy": [_vp],
    "gvx_pvm_info": [_vp, ctypes.POINTER(Dims), ctypes.POINTER(_f), ctypes.POINTER(_vp)],
    "gvx_pvm_clear": [_vp, _vp],
    "gvx_pvm_insert_points": [_vp, _vp, _u64, _u32, _vp, _vp],
    "gvx_dvm_merge_occupied": [_vp, _vp, _vp, _f, _vp],
    "gvx_dvm_extract_distances": [_vp, _vp, ctypes.c_int, _vp],
    "gvx_dvm_init_floodfill": [_vp, _vp, _vp, ctypes.c_int, _vp],
    "gvx_extract_given_distances": [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.POINTER(_u64), _vp],
    "gvx_bvm_collide_types": [_vp, _vp, _vp, _vp, _vp],
    "gvx_bvm_collide_types_pvm": [_vp, _vp, _f, _vp, _vp, _vp],
    "gvx_blist_collide_types_bvm": [_vp, _vp, _i32p, _vp, _vp, _vp],
    "gvx_blist_collide_types_pvm": [_vp, _vp, _f, _i32p, _vp, _vp, _vp],
    "gvx_blist_collide_type_mask_bvm": [_vp, _vp, _vp, _i32p, _vp, _vp],
    "gvx_blist_collide_types_blist": [_vp, _vp, _vp, _vp, _vp],
    "gvx_dvm_write_to_disk": [_vp, ctypes.c_char_p],
    "gvx_dvm_read_from_disk": [_vp, ctypes.c_char_p],
    "gvx_bvm_write_to_disk": [_vp, ctypes.c_char_p],
    "gvx_bvm_read_from_disk": [_vp, ctypes.c_char_p],
    "gvx_pvm_write_to_disk": [_vp, ctypes.c_char_p],
    "gvx_pvm_read_from_disk": [_vp, ctypes.c_char_p],
    "gvx_blist_create": [ctypes.POINTER(Dims), _f, ctypes.POINTER(_vp)],
    "gvx_blist_destroy": [_vp],
    "gvx_blist_size": [_vp, ctypes.POINTER(_u64)],
    "gvx_blist_data": [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)],
    "gvx_blist_clear": [_vp],
    "gvx_blist_insert_points": [_vp, _vp, _u64, _u32, _vp],
    "gvx_blist_set": [_vp, _vp, _vp, _u64, _u32, _vp],
    "gvx_blist_collide_bvm": [_vp, _vp, _i32p, ctypes.c_int, _vp, _vp],
    "gvx_blist_collide_blist": [_vp, _vp, _i32p, _vp, _vp],
    "gvx_lists_collide_bvm": [_vp, _vp, _vp, _u32, _u64, _vp, ctypes.c_int, _vp, _vp],
}
_RESTYPES = {"gvx_last_error": ctypes.c_char_p, "gvx_version": ctypes.c_char_p}

_lib = None


def lib() -> ctypes.CDLL:
    """Load lib/libgvx.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"gvx CUDA library not built: {LIB_PATH} (run `make -C gpu-voxels_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, _st)
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != GVX_OK:
        raise GvxError(status, lib().gvx_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
