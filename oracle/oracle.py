"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (liboracle.so)
and of the reference-kernel build (_ref/libgvref.so).

Only the test suite, the smoke entry and the benchmark's CPU-baseline leg
may import this module; the product never does.  Every function restates a
gpu-voxels routine; see gvx_oracle.c for the file:line each one follows.
The FP64 restatements of the continuous queries (trilinear distance, DH
forward kinematics, sphere clearance, hinge cost) live here in numpy.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

DV_UNINIT = 0x3FFFFFFF
INT_MAX = 2147483647

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def build():
    """Compile liboracle.so (gcc, OpenMP) in place."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


def ref_src():
    """The gpu-voxels source tree (packages/gpu_voxels/src): the environment
    variable GVX_REF_SRC, else the reference checkout beside the repository
    (../reference); None when neither exists."""
    src = os.environ.get("GVX_REF_SRC") or os.path.join(
        os.path.dirname(_HERE), "..", "reference", "packages", "gpu_voxels", "src")
    return os.path.abspath(src) if os.path.isdir(src) else None


def build_ref():
    """Compile _ref/libgvref.so from the reference source tree when present."""
    src = ref_src()
    if src is None:
        return False
    subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF_SRC={src}"], check=True)
    return True


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_coord_to_voxel.argtypes = [ctypes.c_float, ctypes.c_float]
        L.orc_coord_to_voxel.restype = ctypes.c_uint32
        L.orc_dvm_insert.argtypes = [_u32p, _u32p, ctypes.c_float, _f32p, ctypes.c_uint64]
        L.orc_dvm_insert.restype = ctypes.c_int
        L.orc_pba.argtypes = [_u32p, _u32p]
        L.orc_pba.restype = ctypes.c_int
        L.orc_pba_reference_order.argtypes = [_u32p, _u32p]
        L.orc_pba_reference_order.restype = ctypes.c_int
        L.orc_pba_phase1.argtypes = [_u32p, _u32p]
        L.orc_pba_isect.argtypes = [ctypes.c_int] * 8
        L.orc_pba_isect.restype = ctypes.c_float
        L.orc_sqdist.argtypes = [_u32p, _u32p, _u32p, ctypes.c_uint64, _i32p]
        L.orc_dist.argtypes = [_u32p, _u32p, _u32p, ctypes.c_uint64, _i32p]
        L.orc_sqdist_map.argtypes = [_u32p, _u32p, _i32p]
        L.orc_brute_sqdist.argtypes = [_u32p, _u32p, _i32p]
        L.orc_bvm_insert.argtypes = [_u8p, _u32p, ctypes.c_float, _f32p, ctypes.c_uint64, ctypes.c_uint32]
        L.orc_bvm_insert.restype = ctypes.c_int
        L.orc_bvm_clear_bits.argtypes = [_u8p, ctypes.c_uint64, _u8p]
        L.orc_bvm_shift.argtypes = [_u8p, ctypes.c_uint64, ctypes.c_uint32]
        L.orc_bvm_insert_meta_self_coll.argtypes = [_u8p, _u32p, ctypes.c_float, _f32p,
                                                    np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS"),
                                                    ctypes.c_uint32, _u8p, _u8p, _u8p]
        L.orc_bvm_insert_meta_self_coll.restype = ctypes.c_int
        L.orc_bvm_collide.argtypes = [_u8p, _u8p, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int]
        L.orc_bvm_collide.restype = ctypes.c_uint64
        L.orc_bvm_collide_count_omp.argtypes = [_u8p, _u8p, ctypes.c_uint64]
        L.orc_bvm_collide_count_omp.restype = ctypes.c_uint64
        L.orc_list_collide_map.argtypes = [_u32p, _u8p, ctypes.c_uint64, _u8p, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int]
        L.orc_list_collide_map.restype = ctypes.c_uint64
        L.orc_lists_collide_map_omp.argtypes = [_u32p, _u8p, _u64p, ctypes.c_uint64, _u8p, ctypes.c_uint64, _u64p]
        L.orc_list_collide_list.argtypes = [_u32p, ctypes.c_uint64, _u32p, ctypes.c_uint64]
        L.orc_list_collide_list.restype = ctypes.c_uint64
        L.orc_list_insert.argtypes = [_u32p, _u8p, ctypes.POINTER(ctypes.c_uint64), _u32p, ctypes.c_float, _f32p,
                                      ctypes.c_uint64, ctypes.c_uint32]
        _i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
        L.orc_pvm_insert.argtypes = [_i8p, _u32p, ctypes.c_float, _f32p, ctypes.c_uint64, ctypes.c_uint32]
        L.orc_pvm_insert.restype = ctypes.c_int
        L.orc_bvm_collide_pvm.argtypes = [_u8p, _i8p, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int, ctypes.c_int]
        L.orc_bvm_collide_pvm.restype = ctypes.c_uint64
        L.orc_list_collide_pvm.argtypes = [_u32p, _u8p, ctypes.c_uint64, _i8p, ctypes.c_uint64, ctypes.c_int64,
                                           ctypes.c_int, ctypes.c_int]
        L.orc_list_collide_pvm.restype = ctypes.c_uint64
        L.orc_float_to_probability.argtypes = [ctypes.c_float]
        L.orc_float_to_probability.restype = ctypes.c_int
        L.orc_dvm_merge_occupied.argtypes = [_u32p, _i8p, _u32p, _u32p, ctypes.c_float]
        _i16p = np.ctypeslib.ndpointer(dtype=np.int16, flags="C_CONTIGUOUS")
        L.orc_extract_distances.argtypes = [_u32p, _u32p, ctypes.c_int, _i8p]
        L.orc_init_floodfill.argtypes = [_i8p, _i16p, ctypes.c_uint64, ctypes.c_int]
        L.orc_extract_given_distances.argtypes = [_u32p, _u32p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_void_p]
        L.orc_extract_given_distances.restype = ctypes.c_uint64
        L.orc_bvm_collide_types.argtypes = [_u8p, _u8p, ctypes.c_uint64, _u8p]
        L.orc_bvm_collide_types.restype = ctypes.c_uint64
        L.orc_bvm_collide_types_pvm.argtypes = [_u8p, _i8p, ctypes.c_uint64, ctypes.c_float, _u8p]
        L.orc_bvm_collide_types_pvm.restype = ctypes.c_uint64
        L.orc_list_collide_types_map.argtypes = [_u32p, _u8p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                                                 ctypes.c_int, ctypes.c_float, ctypes.c_int64, ctypes.c_void_p,
                                                 ctypes.c_void_p]
        L.orc_list_collide_types_map.restype = ctypes.c_uint64
        L.orc_list_collide_types_list.argtypes = [_u32p, _u8p, ctypes.c_uint64, _u32p, _u8p, ctypes.c_uint64, _u8p]
        L.orc_list_collide_types_list.restype = ctypes.c_uint64
        L.orc_num_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's own kernels (GPU), or None when not built / no GPU."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libgvref.so")
        if not os.path.exists(path):
            return None
        R = ctypes.CDLL(path)
        R.ref_available.restype = ctypes.c_int
        R.ref_pba.argtypes = [_u32p, _u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        R.ref_pba.restype = ctypes.c_int
        R.ref_pba_time.argtypes = [_u32p, _u32p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
        R.ref_pba_time.restype = ctypes.c_int
        R.ref_dvm_insert.argtypes = [_u32p, _u32p, ctypes.c_float, _f32p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int)]
        R.ref_dvm_insert.restype = ctypes.c_int
        R.ref_bvm_collide.argtypes = [_u8p, _u8p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)]
        R.ref_bvm_collide.restype = ctypes.c_int
        R.ref_lists_collide_map.argtypes = [_u32p, _u8p, _u64p, ctypes.c_uint32, _u8p, _u32p,
                                            np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS"), _u64p]
        R.ref_lists_collide_map.restype = ctypes.c_int
        _i8 = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
        _i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        R.ref_bvm_collide_pvm.argtypes = [_u8p, _i8, ctypes.c_uint32, ctypes.c_float, ctypes.POINTER(ctypes.c_uint64)]
        R.ref_bvm_collide_pvm.restype = ctypes.c_int
        R.ref_list_collide_pvm.argtypes = [_u32p, _u8p, ctypes.c_uint32, _i8, _u32p, _i32, ctypes.c_float,
                                           ctypes.POINTER(ctypes.c_uint64)]
        R.ref_list_collide_pvm.restype = ctypes.c_int
        _REF = R
    return _REF


def num_threads() -> int:
    return lib().orc_num_threads()


def _dims(dims):
    return np.ascontiguousarray(np.asarray(dims, dtype=np.uint32))


def _pts(xyz):
    return np.ascontiguousarray(np.asarray(xyz, dtype=np.float32).reshape(-1, 3))


# ---- DistanceVoxelMap ------------------------------------------------------

def dvm_empty(dims) -> np.ndarray:
    """clearMap: every voxel uninitialised (flat uint32, x fastest)."""
    return np.full(int(np.prod(np.asarray(dims, dtype=np.int64))), DV_UNINIT, dtype=np.uint32)


def dvm_insert(vmap: np.ndarray, dims, side: float, xyz) -> bool:
    """kernelInsertGlobalPointCloud<DistanceVoxel>; returns the outside flag."""
    p = _pts(xyz)
    return bool(lib().orc_dvm_insert(vmap, _dims(dims), np.float32(side), p, p.shape[0]))


def pba(vmap: np.ndarray, dims) -> np.ndarray:
    """parallelBanding3D(1,1,1) for any dims, in place; returns vmap."""
    rc = lib().orc_pba(vmap, _dims(dims))
    if rc != 0:
        raise ValueError(f"oracle pba rejected dims {dims}")
    return vmap


def pba_reference_order(vmap: np.ndarray, dims) -> np.ndarray:
    """Literal launch order of parallelBanding3D (needs dims x == y)."""
    rc = lib().orc_pba_reference_order(vmap, _dims(dims))
    if rc != 0:
        raise ValueError("reference order needs x == y")
    return vmap


def phase1(vmap: np.ndarray, dims) -> np.ndarray:
    lib().orc_pba_phase1(vmap, _dims(dims))
    return vmap


def sqdist(vmap, dims, ids) -> np.ndarray:
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    out = np.empty(ids.shape[0], dtype=np.int32)
    lib().orc_sqdist(vmap, _dims(dims), ids, ids.shape[0], out)
    return out


def dist(vmap, dims, ids) -> np.ndarray:
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    out = np.empty(ids.shape[0], dtype=np.int32)
    lib().orc_dist(vmap, _dims(dims), ids, ids.shape[0], out)
    return out


def sqdist_map(vmap, dims) -> np.ndarray:
    out = np.empty(vmap.shape[0], dtype=np.int32)
    lib().orc_sqdist_map(vmap, _dims(dims), out)
    return out


def brute_sqdist(inserted, dims) -> np.ndarray:
    out = np.empty(inserted.shape[0], dtype=np.int32)
    lib().orc_brute_sqdist(np.ascontiguousarray(inserted, dtype=np.uint32), _dims(dims), out)
    return out


def coord_to_voxel(c: float, side: float) -> int:
    return int(lib().orc_coord_to_voxel(float(c), float(side)))


def isect(*args) -> float:
    return float(lib().orc_pba_isect(*[int(a) for a in args]))


# ---- BitVoxel maps and lists ----------------------------------------------

def bvm_empty(dims) -> np.ndarray:
    return np.zeros(int(np.prod(np.asarray(dims, dtype=np.int64))) * 32, dtype=np.uint8)


def bvm_insert(bmap: np.ndarray, dims, side: float, xyz, meaning: int) -> bool:
    p = _pts(xyz)
    return bool(lib().orc_bvm_insert(bmap, _dims(dims), np.float32(side), p, p.shape[0], int(meaning)))


EBVM_SWEPT_VOLUME_START = 4  # GV/helpers/common_defines.h:57


def bvm_clear_bits(bmap: np.ndarray, bits) -> np.ndarray:
    """BitVoxelMap::clearBits on a flat uint8 map (32 bytes per voxel), in place."""
    lib().orc_bvm_clear_bits(bmap, bmap.shape[0] // 32, np.ascontiguousarray(np.asarray(bits, np.uint8).reshape(32)))
    return bmap


def bvm_shift(bmap: np.ndarray, shift: int) -> np.ndarray:
    """BitVoxelMap::shiftLeftSweptVolumeIDs (performLeftShift per voxel), in place."""
    lib().orc_bvm_shift(bmap, bmap.shape[0] // 32, int(shift))
    return bmap


def default_self_coll_masks(meanings) -> np.ndarray:
    """insertMetaPointCloudWithSelfCollisionCheck's default masks (BitVoxelMap.hpp:
    278-293): every bit but eBVM_COLLISION and the sub-cloud's own meaning."""
    masks = np.full((len(meanings), 32), 0xFF, dtype=np.uint8)
    for k, m in enumerate(meanings):
        masks[k, 0] &= ~np.uint8(1 << 2)
        masks[k, m >> 3] &= ~np.uint8(1 << (m & 7))
    return masks


def bvm_insert_meta_self_coll(bmap: np.ndarray, dims, side: float, clouds, meanings=None, masks=None):
    """BitVoxelMap::insertMetaPointCloudWithSelfCollisionCheck; returns
    (self_collision, colliding uint8[32], outside)."""
    parts = [_pts(c) for c in clouds]
    offsets = np.zeros(len(parts) + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum([q.shape[0] for q in parts])
    xyz = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros((0, 3), np.float32), dtype=np.float32)
    mean = np.asarray([EBVM_SWEPT_VOLUME_START + k for k in range(len(parts))] if meanings is None else meanings,
                      dtype=np.uint8)
    msk = default_self_coll_masks(mean) if masks is None else np.ascontiguousarray(masks, dtype=np.uint8).reshape(-1, 32)
    colliding = np.zeros(32, dtype=np.uint8)
    out = lib().orc_bvm_insert_meta_self_coll(bmap, _dims(dims), np.float32(side), xyz, offsets, len(parts),
                                              np.ascontiguousarray(mean), np.ascontiguousarray(msk), colliding)
    return bool(colliding.any()), colliding, bool(out)


def bvm_collide(self_map: np.ndarray, other: np.ndarray, offset_linear: int = 0, mark: bool = True) -> int:
    n = self_map.shape[0] // 32
    return int(lib().orc_bvm_collide(self_map, other, n, int(offset_linear), 1 if mark else 0))


def bvm_collide_count_omp(self_map: np.ndarray, other: np.ndarray) -> int:
    return int(lib().orc_bvm_collide_count_omp(self_map, other, self_map.shape[0] // 32))


def list_collide_map(ids, list_vox: np.ndarray, bmap: np.ndarray, offset_linear: int = 0, mark: bool = True) -> int:
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    return int(lib().orc_list_collide_map(ids, list_vox, ids.shape[0], bmap, bmap.shape[0] // 32, int(offset_linear),
                                          1 if mark else 0))


def lists_collide_map_omp(ids, list_vox, offsets, bmap) -> np.ndarray:
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    counts = np.zeros(offsets.shape[0] - 1, dtype=np.uint64)
    lib().orc_lists_collide_map_omp(np.ascontiguousarray(ids, dtype=np.uint32), list_vox, offsets, counts.shape[0], bmap,
                                    bmap.shape[0] // 32, counts)
    return counts


def list_collide_list(a, b) -> int:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    return int(lib().orc_list_collide_list(a, a.shape[0], b, b.shape[0]))


def list_insert(ids, vox, dims, side, xyz, meaning):
    """TemplateVoxelList::insertPointCloud; returns new (ids, voxels)."""
    p = _pts(xyz)
    n0 = 0 if ids is None else int(ids.shape[0])
    cap = n0 + p.shape[0] + 1
    ids_io = np.zeros(cap, dtype=np.uint32)
    vox_io = np.zeros(cap * 32, dtype=np.uint8)
    if n0:
        ids_io[:n0] = ids
        vox_io[: n0 * 32] = vox
    n = ctypes.c_uint64(n0)
    lib().orc_list_insert(ids_io, vox_io, ctypes.byref(n), _dims(dims), np.float32(side), p, p.shape[0], int(meaning))
    return ids_io[: n.value].copy(), vox_io[: n.value * 32].copy()


# ---- FP64 continuous queries ------------------------------------------------

def pvm_empty(dims) -> np.ndarray:
    """ProbVoxelMap after clearMap: every voxel UNKNOWN (-128)."""
    return np.full(int(np.prod(dims)), -128, dtype=np.int8)


def pvm_insert(pmap: np.ndarray, dims, side: float, xyz, meaning: int) -> bool:
    p = _pts(xyz)
    return bool(lib().orc_pvm_insert(pmap, _dims(dims), np.float32(side), p, p.shape[0], int(meaning)))


def float_to_probability(val: float) -> int:
    return int(lib().orc_float_to_probability(float(val)))


def bvm_collide_pvm(self_map: np.ndarray, pmap: np.ndarray, coll_threshold: float = 1.0, offset_linear: int = 0,
                    mark: bool = True) -> int:
    """BitVoxelMap::collideWith(const ProbVoxelMap*): marks self_map in place."""
    return int(lib().orc_bvm_collide_pvm(self_map, pmap, pmap.shape[0], int(offset_linear),
                                         float_to_probability(coll_threshold), 1 if mark else 0))


def list_collide_pvm(ids, list_vox: np.ndarray, pmap: np.ndarray, coll_threshold: float = 1.0, offset_linear: int = 0,
                     mark: bool = True) -> int:
    """BitVoxelList::collideWith(const ProbVoxelMap*): marks list_vox in place."""
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    return int(lib().orc_list_collide_pvm(ids, list_vox, ids.shape[0], pmap, pmap.shape[0], int(offset_linear),
                                          float_to_probability(coll_threshold), 1 if mark else 0))


def dvm_merge_occupied(vmap: np.ndarray, pmap: np.ndarray, dims, offset=(0, 0, 0), threshold: float = 0.5) -> None:
    lib().orc_dvm_merge_occupied(vmap, pmap, _dims(dims), np.asarray(offset, dtype=np.uint32), float(threshold))


def extract_distances(vmap: np.ndarray, dims, robot_radius: int = 0) -> np.ndarray:
    out = np.empty(vmap.size, dtype=np.int8)
    lib().orc_extract_distances(vmap, _dims(dims), int(robot_radius), out)
    return out


def init_floodfill(dist: np.ndarray, robot_radius: int) -> np.ndarray:
    out = np.empty(dist.size, dtype=np.int16)
    lib().orc_init_floodfill(np.ascontiguousarray(dist, dtype=np.int8), out, dist.size, int(robot_radius))
    return out


def extract_given_distances(vmap: np.ndarray, dims, min_dist: int, max_dist: int):
    """-> (ids uint32[k], voxels uint8[k*32])"""
    k = int(lib().orc_extract_given_distances(vmap, _dims(dims), int(min_dist), int(max_dist), None, None))
    ids = np.empty(max(k, 1), dtype=np.uint32)
    vox = np.empty(max(k, 1) * 32, dtype=np.uint8)
    lib().orc_extract_given_distances(vmap, _dims(dims), int(min_dist), int(max_dist), ids.ctypes.data, vox.ctypes.data)
    return ids[:k], vox[:k * 32]


def bvm_collide_types(self_map: np.ndarray, other: np.ndarray):
    """-> (count, types uint8[32]); marks self."""
    types = np.zeros(32, dtype=np.uint8)
    n = lib().orc_bvm_collide_types(self_map, other, self_map.size // 32, types)
    return int(n), types


def bvm_collide_types_pvm(self_map: np.ndarray, pmap: np.ndarray, threshold: float):
    types = np.zeros(32, dtype=np.uint8)
    n = lib().orc_bvm_collide_types_pvm(self_map, pmap, self_map.size // 32, float(threshold), types)
    return int(n), types


def list_collide_types_map(ids, list_vox: np.ndarray, bmap: np.ndarray, offset_linear: int = 0, mask=None,
                           prob_threshold: float = None):
    """List vs BitVoxel map (bmap uint8, 32 B voxels) or, with prob_threshold,
    vs a ProbVoxelMap (bmap int8).  -> (count, types uint8[32]); marks the list."""
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    types = np.zeros(32, dtype=np.uint8)
    kind = 0 if prob_threshold is None else 1
    map_n = bmap.size // 32 if kind == 0 else bmap.size
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    n = lib().orc_list_collide_types_map(ids, list_vox, ids.size, bmap.ctypes.data, map_n, kind,
                                         float(prob_threshold or 0.0), int(offset_linear),
                                         None if m is None else m.ctypes.data, types.ctypes.data)
    return int(n), types


def list_collide_types_list(ids_a, vox_a, ids_b, vox_b):
    types = np.zeros(32, dtype=np.uint8)
    a = np.ascontiguousarray(ids_a, dtype=np.uint32)
    b = np.ascontiguousarray(ids_b, dtype=np.uint32)
    n = lib().orc_list_collide_types_list(a, np.ascontiguousarray(vox_a), a.size, b, np.ascontiguousarray(vox_b), b.size,
                                          types)
    return int(n), types


def decode_sites(vmap: np.ndarray):
    v = vmap.astype(np.int64)
    return v & 0x3FF, (v >> 10) & 0x3FF, v >> 20


def corner_dist64(vmap: np.ndarray, dims, i, j, k) -> np.ndarray:
    """sqrt(squaredObstacleDistance) at lattice points, float64, voxel units."""
    X, Y, _ = (int(d) for d in dims)
    v = vmap[(k.astype(np.int64) * Y + j) * X + i].astype(np.int64)
    ox, oy, oz = v & 0x3FF, (v >> 10) & 0x3FF, v >> 20
    sq = (i - ox) ** 2 + (j - oy) ** 2 + (k - oz) ** 2
    bad = (ox == 1023) | (oy == 1023) | (oz == 1023)
    sq = np.where(bad, INT_MAX, sq)
    return np.sqrt(sq.astype(np.float64))


def trilinear64(vmap: np.ndarray, dims, side: float, xyz):
    """FP64 trilinear distance (metres) and gradient at float points, with the
    same lattice, clamping and corner convention as the CUDA queries."""
    p = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    side = float(np.float32(side))
    idx, frac, free = [], [], []
    for a in range(3):
        n = int(dims[a])
        u = p[:, a] / side - 0.5
        fr = (u >= 0) & (u <= n - 1)
        uc = np.clip(np.nan_to_num(u, nan=0.0), 0, n - 1)
        i0 = np.minimum(np.floor(uc).astype(np.int64), max(n - 2, 0))
        i1 = np.minimum(i0 + 1, n - 1)
        idx.append((i0, i1))
        frac.append(uc - i0)
        free.append(fr)
    (i0, i1), (j0, j1), (k0, k1) = idx
    fx, fy, fz = frac
    D = {}
    for a, ii in (("0", i0), ("1", i1)):
        for b, jj in (("0", j0), ("1", j1)):
            for c, kk in (("0", k0), ("1", k1)):
                D[a + b + c] = corner_dist64(vmap, dims, ii, jj, kk)
    e00 = D["000"] + fx * (D["100"] - D["000"])
    e10 = D["010"] + fx * (D["110"] - D["010"])
    e01 = D["001"] + fx * (D["101"] - D["001"])
    e11 = D["011"] + fx * (D["111"] - D["011"])
    g0 = e00 + fy * (e10 - e00)
    g1 = e01 + fy * (e11 - e01)
    d = g0 + fz * (g1 - g0)
    sx0 = (D["100"] - D["000"]) + fy * ((D["110"] - D["010"]) - (D["100"] - D["000"]))
    sx1 = (D["101"] - D["001"]) + fy * ((D["111"] - D["011"]) - (D["101"] - D["001"]))
    gx = np.where(free[0], sx0 + fz * (sx1 - sx0), 0.0)
    gy = np.where(free[1], (e10 - e00) + fz * ((e11 - e01) - (e10 - e00)), 0.0)
    gz = np.where(free[2], g1 - g0, 0.0)
    return d * side, np.stack([gx, gy, gz], axis=1)


def dh_matrix64(theta, d, a, alpha, q):
    """DHParameters::convertDHtoM (GV/robot/dh_robot/KinematicLink.cu:24-79),
    revolute joint, float64: Rz(theta+q) Tz(d) Tx(a) Rx(alpha)."""
    ct, st = np.cos(theta + q), np.sin(theta + q)
    ca, sa = np.cos(alpha), np.sin(alpha)
    m = np.zeros(q.shape + (4, 4))
    m[..., 0, 0], m[..., 0, 1], m[..., 0, 2], m[..., 0, 3] = ct, -st * ca, st * sa, a * ct
    m[..., 1, 0], m[..., 1, 1], m[..., 1, 2], m[..., 1, 3] = st, ct * ca, -ct * sa, a * st
    m[..., 2, 1], m[..., 2, 2], m[..., 2, 3] = sa, ca, d
    m[..., 3, 3] = 1.0
    return m


def sphere_centres64(arm: dict, q: np.ndarray) -> np.ndarray:
    """Chain as KinematicChain::setConfiguration (KinematicChain.cu:104-124):
    link j spans the origins of F_j = base*A_0*...*A_{j-1} and F_{j+1}."""
    q = np.asarray(q, dtype=np.float64)
    J = arm["n_joints"]
    # every arm parameter as the device holds it (float32), then FP64
    F = np.broadcast_to(np.asarray(arm["base"], dtype=np.float32).astype(np.float64).reshape(4, 4),
                        q.shape[:-1] + (4, 4)).copy()
    origins = [F[..., :3, 3].copy()]
    for j in range(J):
        A = dh_matrix64(float(np.float32(arm["theta"][j])), float(np.float32(arm["d"][j])),
                        float(np.float32(arm["a"][j])), float(np.float32(arm["alpha"][j])), q[..., j])
        F = F @ A
        origins.append(F[..., :3, 3].copy())
    O = np.stack(origins, axis=-2)  # [..., J+1, 3]
    link = np.asarray(arm["link"], dtype=np.int64)
    t = np.asarray(arm["t"], dtype=np.float32).astype(np.float64)[:, None]
    return O[..., link, :] + t * (O[..., link + 1, :] - O[..., link, :])


def sphere_clearance64(vmap, dims, side, arm, q) -> np.ndarray:
    c = sphere_centres64(arm, q)
    shp = c.shape
    d, _ = trilinear64(vmap, dims, side, c.reshape(-1, 3))
    r = np.asarray(arm["r"], dtype=np.float32).astype(np.float64)
    return (d.reshape(shp[:-1]) - r).min(axis=-1)


def traj_cost64(vmap, dims, side, arm, q, margin) -> np.ndarray:
    """q: [n_traj, n_wp, J] -> cost per trajectory (FP64)."""
    c = sphere_centres64(arm, q)
    shp = c.shape
    d, _ = trilinear64(vmap, dims, side, c.reshape(-1, 3))
    r = np.asarray(arm["r"], dtype=np.float32).astype(np.float64)
    clear = d.reshape(shp[:-1]) - r
    return np.maximum(0.0, float(np.float32(margin)) - clear).sum(axis=(-1, -2))


def arm_frames64(arm: dict, q: np.ndarray):
    """FP64 chain of KinematicChain::setConfiguration (KinematicChain.cu:104-124):
    -> (origins o_0..o_J [..., J+1, 3], joint axes z_0..z_{J-1} [..., J, 3]);
    joint j turns about z_j (third column of F_j) through o_j."""
    q = np.asarray(q, dtype=np.float64)
    J = arm["n_joints"]
    F = np.broadcast_to(np.asarray(arm["base"], dtype=np.float32).astype(np.float64).reshape(4, 4),
                        q.shape[:-1] + (4, 4)).copy()
    origins, axes = [F[..., :3, 3].copy()], []
    for j in range(J):
        axes.append(F[..., :3, 2].copy())
        A = dh_matrix64(float(np.float32(arm["theta"][j])), float(np.float32(arm["d"][j])),
                        float(np.float32(arm["a"][j])), float(np.float32(arm["alpha"][j])), q[..., j])
        F = F @ A
        origins.append(F[..., :3, 3].copy())
    return np.stack(origins, axis=-2), np.stack(axes, axis=-2)


def traj_cost_grad64(vmap, dims, side, arm, q, margin, gcost):
    """Analytic FP64 adjoint of traj_cost64 (TEST INFRASTRUCTURE).

    For an active sphere s (margin - (d(c_s) - r_s) > 0) on link j,
    d cost / d q_k = -grad d(c_s) . (z_k x (c_s - o_k)) for every k <= j.
    Returns (grad [B, W, J] = gcost[b] * d cost_b / d q, scale [B, W, J] =
    gcost[b] * sum over active spheres on links >= k of |z_k x (c_s - o_k)|_1,
    gap [B, W] = the smallest |margin - clearance| of the waypoint's spheres).
    `scale` times a bound on the spatial gradient's component error bounds the
    adjoint's error; `gap` tells waypoints whose active set a rounding could flip.
    """
    q = np.asarray(q, dtype=np.float64)
    B, W, J = q.shape
    O, Z = arm_frames64(arm, q)                                   # [B,W,J+1,3], [B,W,J,3]
    link = np.asarray(arm["link"], dtype=np.int64)
    t = np.asarray(arm["t"], dtype=np.float32).astype(np.float64)[:, None]
    C = O[..., link, :] + t * (O[..., link + 1, :] - O[..., link, :])   # [B,W,S,3]
    d, g = trilinear64(vmap, dims, side, C.reshape(-1, 3))
    S = C.shape[2]
    d = d.reshape(B, W, S)
    g = g.reshape(B, W, S, 3)
    r = np.asarray(arm["r"], dtype=np.float32).astype(np.float64)
    m = float(np.float32(margin))
    gap_all = m - (d - r)
    active = gap_all > 0
    gc = np.asarray(gcost, dtype=np.float64)[:, None, None]
    grad = np.zeros((B, W, J))
    scale = np.zeros((B, W, J))
    for k in range(J):
        on = active & (link[None, None, :] >= k)                   # spheres moved by joint k
        lever = np.cross(Z[..., k, None, :], C - O[..., k, None, :])  # z_k x (c_s - o_k)
        grad[..., k] = -(np.einsum("bwsi,bwsi->bws", g, lever) * on).sum(-1)
        scale[..., k] = (np.abs(lever).sum(-1) * on).sum(-1)
    return grad * gc, scale * gc, np.abs(gap_all).min(-1)
