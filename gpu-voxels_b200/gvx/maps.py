"""Python handles over the C ABI, named after gpu-voxels' map classes.

DistanceVoxelMap, BitVectorVoxelMap and BitVectorVoxelList expose the
reference's method names (clearMap, insertPointCloud, parallelBanding3D,
getSquaredDistances, collideWith, ...) with torch CUDA tensors as device
buffers.  Every call goes to lib/libgvx.so on the current torch stream.
Methods that the reference makes blocking (the *ToHost queries and the
collideWith counts) synchronise here too.
"""
from __future__ import annotations

import ctypes
from typing import Iterable, Optional, Sequence

import numpy as np
import torch

from . import _abi
from ._abi import Arm, Dims, call

BIT_VECTOR_LENGTH = 256
eBVM_FREE = 0
eBVM_OCCUPIED = 1
eBVM_COLLISION = 2


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: Optional[torch.Tensor]) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def _dev_points(points) -> torch.Tensor:
    t = points if isinstance(points, torch.Tensor) else torch.as_tensor(points)
    t = t.to(device="cuda", dtype=torch.float32).reshape(-1, 3).contiguous()
    return t


def _dev_u32(ids) -> torch.Tensor:
    t = ids if isinstance(ids, torch.Tensor) else torch.as_tensor(ids, dtype=torch.int64)
    if t.dtype != torch.int32:
        t = t.to(torch.int64).to(torch.int32)  # same 32 bits
    return t.to("cuda").contiguous()


def _check_clone(dst, src) -> None:
    """TemplateVoxelMap::clone (GV/voxelmap/TemplateVoxelMap.hpp:1101-1120) copies
    only between maps of equal dims and voxel side length."""
    if dst.dims != src.dims or np.float32(dst.voxel_side_length) != np.float32(src.voxel_side_length):
        raise ValueError(f"clone: dims {src.dims} / side {src.voxel_side_length} differ from "
                         f"{dst.dims} / {dst.voxel_side_length}")


def _offset(offset: Sequence[int]) -> ctypes.Array:
    o = (ctypes.c_int32 * 3)(*[int(v) for v in offset])
    return o


class DistanceVoxelMap:
    """DistanceVoxelMap (GV/voxelmap/DistanceVoxelMap.h): uint32 sites per voxel."""

    def __init__(self, dims: Sequence[int], voxel_side_length: float, voxels: Optional[torch.Tensor] = None):
        self.dims = tuple(int(d) for d in dims)
        self.voxel_side_length = float(voxel_side_length)
        h = ctypes.c_void_p()
        d = Dims(*self.dims)
        self._owner = None
        if voxels is None:
            call("gvx_dvm_create", ctypes.byref(d), self.voxel_side_length, ctypes.byref(h))
        else:
            assert voxels.is_cuda and voxels.dtype == torch.int32 and voxels.numel() == self.size
            self._owner = voxels
            call("gvx_dvm_wrap", ctypes.byref(d), self.voxel_side_length, _ptr(voxels), ctypes.byref(h))
        self._h = h
        self._destroy = _abi.lib().gvx_dvm_destroy

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            # bound at creation: module globals may already be gone at interpreter exit
            getattr(self, "_destroy", None) and self._destroy(h)
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def size(self) -> int:
        return self.dims[0] * self.dims[1] * self.dims[2]

    def clone(self, other: "DistanceVoxelMap") -> None:
        """Copy `other`'s voxels (equal dims and side length; stream-ordered)."""
        _check_clone(self, other)
        if other is not self:
            self.data().copy_(other.data())

    def data(self) -> torch.Tensor:
        """Borrowed int32 CUDA view of the voxel buffer (bit pattern = uint32
        sites); valid while this map is alive."""
        if self._owner is not None:
            return self._owner
        d, s, p = Dims(), ctypes.c_float(), ctypes.c_void_p()
        call("gvx_dvm_info", self._h, ctypes.byref(d), ctypes.byref(s), ctypes.byref(p))
        return _device_view(p.value, self.size)

    def writeToDisk(self, path: str) -> None:
        """TemplateVoxelMap::writeToDisk: the reference's binary map file."""
        call("gvx_dvm_write_to_disk", self._h, str(path).encode())

    def readFromDisk(self, path: str) -> None:
        """TemplateVoxelMap::readFromDisk (type and dims must match)."""
        call("gvx_dvm_read_from_disk", self._h, str(path).encode())

    def clearMap(self) -> None:
        call("gvx_dvm_clear", self._h, _stream())

    def insertPointCloud(self, points, meaning: int = eBVM_OCCUPIED, outside: Optional[torch.Tensor] = None) -> None:
        p = _dev_points(points)
        call("gvx_dvm_insert_points", self._h, _ptr(p), p.shape[0], _ptr(outside), _stream())

    def extract_distances(self, robot_radius: int = 0, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """int8 free-space byte per voxel (DistanceVoxelMap::extract_distances)."""
        out = torch.empty(self.size, dtype=torch.int8, device="cuda") if out is None else out
        call("gvx_dvm_extract_distances", self._h, _ptr(out), int(robot_radius), _stream())
        return out

    def init_floodfill(self, distances: torch.Tensor, robot_radius: int) -> torch.Tensor:
        """int16 per voxel: 32765 where distances <= robot_radius, else 32767."""
        out = torch.empty(self.size, dtype=torch.int16, device="cuda")
        call("gvx_dvm_init_floodfill", self._h, _ptr(distances), _ptr(out), int(robot_radius), _stream())
        return out

    def mergeOccupied(self, other: "ProbVoxelMap", voxel_offset=(0, 0, 0), occupancy_threshold: float = 0.5) -> None:
        """Voxels of `other` above the threshold become sites (own coordinates + offset)."""
        off = (ctypes.c_uint32 * 3)(*[int(v) & 0xFFFFFFFF for v in voxel_offset])
        call("gvx_dvm_merge_occupied", self._h, other.handle, off, float(occupancy_threshold), _stream())

    def voxelize_edt(self, points, outside: Optional[torch.Tensor] = None) -> None:
        """clearMap + insertPointCloud + parallelBanding3D in one call (same result)."""
        p = _dev_points(points)
        call("gvx_dvm_voxelize_edt", self._h, _ptr(p), p.shape[0], _ptr(outside), _stream())

    def parallelBanding3D(self, m1: int = 1, m2: int = 1, m3: int = 1, *unused) -> None:
        call("gvx_dvm_edt", self._h, m1, m2, m3, _stream())

    def edt_pass(self, pass_index: int) -> None:
        """One EDT stage: 0 = z sweep, 1 = y sweep, 2 = x sweep, 3 = y and x
        sweeps as the one fused launch parallelBanding3D uses."""
        call("gvx_dvm_edt_pass", self._h, int(pass_index), _stream())

    def autotune(self, force: bool = False) -> dict:
        """Pick the fastest EDT sweep configuration for this map (timed on a
        copy of its current content; cached per device and dims, and across
        processes through the file named by GVX_TUNE_CACHE)."""
        c = _abi.EdtConfig()
        call("gvx_dvm_autotune", self._h, int(bool(force)), ctypes.byref(c), _stream())
        return {"rows": c.rows, "fused": c.fused, "ms": c.ms}

    def set_edt_config(self, rows: int = 0, fused: int = 1) -> None:
        """Fix the EDT sweep configuration (rows 16 or 32, 0 = default; fused 0/1)."""
        c = _abi.EdtConfig(rows, fused, 0.0)
        call("gvx_dvm_set_edt_config", self._h, ctypes.byref(c))

    def edt_check(self) -> int:
        """Synchronise and return the error word of the last EDT (0 = ok);
        raises GvxError (GVX_ERR_TIMEOUT) when a bounded wait gave up."""
        flags = ctypes.c_uint32(0)
        call("gvx_dvm_edt_check", self._h, ctypes.byref(flags))
        return int(flags.value)

    def getSquaredDistances(self, ids: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        ids = _dev_u32(ids)
        out = torch.empty(ids.shape[0], dtype=torch.int32, device="cuda") if out is None else out
        call("gvx_dvm_sqdist", self._h, _ptr(ids), ids.shape[0], _ptr(out), _stream())
        return out

    def getSquaredDistancesToHost(self, ids) -> list:
        return self.getSquaredDistances(ids).cpu().tolist()

    def getDistances(self, ids: torch.Tensor) -> torch.Tensor:
        ids = _dev_u32(ids)
        out = torch.empty(ids.shape[0], dtype=torch.int32, device="cuda")
        call("gvx_dvm_dist", self._h, _ptr(ids), ids.shape[0], _ptr(out), _stream())
        return out

    def getDistancesToHost(self, ids) -> list:
        return self.getDistances(ids).cpu().tolist()

    def gatherVoxelsByIndex(self, ids) -> torch.Tensor:
        ids = _dev_u32(ids)
        out = torch.empty(ids.shape[0], dtype=torch.int32, device="cuda")
        call("gvx_dvm_gather", self._h, _ptr(ids), ids.shape[0], _ptr(out), _stream())
        return out

    def squaredDistanceMap(self) -> torch.Tensor:
        out = torch.empty(self.size, dtype=torch.int32, device="cuda")
        call("gvx_dvm_sqdist_map", self._h, _ptr(out), _stream())
        return out

    def getSquaredObstacleDistance(self, x: int, y: int, z: int) -> int:
        return self.getSquaredDistancesToHost([(z * self.dims[1] + y) * self.dims[0] + x])[0]

    # continuous queries (new)
    def trilinear(self, points: torch.Tensor, with_grad: bool = True):
        p = _dev_points(points)
        n = p.shape[0]
        dist = torch.empty(n, dtype=torch.float32, device="cuda")
        grad = torch.empty(n, 3, dtype=torch.float32, device="cuda") if with_grad else None
        call("gvx_query_trilinear", self._h, _ptr(p), n, _ptr(dist), _ptr(grad), _stream())
        return (dist, grad) if with_grad else dist

    def autotune_queries(self, points: torch.Tensor, with_grad: bool = True, force: bool = False) -> dict:
        """Pick the fastest launch shape of the trilinear query kernels, timed on
        `points` against this map (cached per device for the process); applies
        to every map's queries and to the batched query."""
        p = _dev_points(points)
        n = p.shape[0]
        dist = torch.empty(n, dtype=torch.float32, device="cuda")
        grad = torch.empty(n, 3, dtype=torch.float32, device="cuda") if with_grad else None
        c = _abi.QueryConfig()
        call("gvx_query_autotune", self._h, _ptr(p), n, _ptr(dist), _ptr(grad), int(bool(force)), ctypes.byref(c),
             _stream())
        return {"threads": c.threads, "blocks_per_sm": c.blocks_per_sm, "ms": c.ms}

    def trilinear_backward(self, points: torch.Tensor, grad_dist: torch.Tensor) -> torch.Tensor:
        p = _dev_points(points)
        g = grad_dist.to(device="cuda", dtype=torch.float32).contiguous()
        out = torch.empty(p.shape[0], 3, dtype=torch.float32, device="cuda")
        call("gvx_query_trilinear_bwd", self._h, _ptr(p), p.shape[0], _ptr(g), _ptr(out), _stream())
        return out

    def sphere_clearance(self, arm: Arm, q: torch.Tensor) -> torch.Tensor:
        q = q.to(device="cuda", dtype=torch.float32).contiguous()
        n = q.shape[0]
        out = torch.empty(n, dtype=torch.float32, device="cuda")
        call("gvx_sphere_clearance", self._h, ctypes.byref(arm), _ptr(q), n, _ptr(out), _stream())
        return out

    def traj_cost(self, arm: Arm, q: torch.Tensor, margin: float) -> torch.Tensor:
        q = q.to(device="cuda", dtype=torch.float32).contiguous()
        out = torch.empty(q.shape[0], dtype=torch.float32, device="cuda")
        call("gvx_traj_cost", self._h, ctypes.byref(arm), _ptr(q), q.shape[0], q.shape[1], float(margin), _ptr(out),
             _stream())
        return out

    def traj_cost_backward(self, arm: Arm, q: torch.Tensor, margin: float, grad_cost: torch.Tensor) -> torch.Tensor:
        q = q.to(device="cuda", dtype=torch.float32).contiguous()
        g = grad_cost.to(device="cuda", dtype=torch.float32).contiguous()
        out = torch.empty_like(q)
        call("gvx_traj_cost_bwd", self._h, ctypes.byref(arm), _ptr(q), q.shape[0], q.shape[1], float(margin), _ptr(g),
             _ptr(out), _stream())
        return out


def _device_view(ptr: int, n: int) -> torch.Tensor:
    """A borrowed int32 CUDA tensor over n elements at a raw device pointer."""
    class _CAI:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_CAI(), device="cuda")


def _device_view_u8(ptr: int, n: int) -> torch.Tensor:
    class _CAI:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_CAI(), device="cuda")


def _device_view_i8(ptr: int, n: int) -> torch.Tensor:
    class _CAI:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "|i1", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_CAI(), device="cuda")


def extract_given_distances(dist_map: "DistanceVoxelMap", min_dist: int, max_dist: int,
                            result: "BitVectorVoxelList") -> int:
    """distance_map_converter::extract_given_distances: voxels whose free-space
    byte lies in [min_dist, max_dist] become `result` (blocking; returns the count)."""
    n = ctypes.c_uint64(0)
    call("gvx_extract_given_distances", dist_map.handle, int(min_dist), int(max_dist), result.handle, ctypes.byref(n),
         _stream())
    return int(n.value)


class ProbVoxelMap:
    """ProbVoxelMap (GV/voxelmap/ProbVoxelMap.h): one int8 occupancy per voxel
    (-128 unknown, -127..127 log-odds-like probability)."""

    def __init__(self, dims: Sequence[int], voxel_side_length: float):
        self.dims = tuple(int(d) for d in dims)
        self.voxel_side_length = float(voxel_side_length)
        h = ctypes.c_void_p()
        call("gvx_pvm_create", ctypes.byref(Dims(*self.dims)), self.voxel_side_length, ctypes.byref(h))
        self._h = h
        self._destroy = _abi.lib().gvx_pvm_destroy

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            getattr(self, "_destroy", None) and self._destroy(h)
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def size(self) -> int:
        return self.dims[0] * self.dims[1] * self.dims[2]

    def clone(self, other: "ProbVoxelMap") -> None:
        """Copy `other`'s occupancies (equal dims and side length; stream-ordered)."""
        _check_clone(self, other)
        if other is not self:
            self.data().copy_(other.data())

    def data(self) -> torch.Tensor:
        """Borrowed int8 CUDA view of the occupancies."""
        d, s, p = Dims(), ctypes.c_float(), ctypes.c_void_p()
        call("gvx_pvm_info", self._h, ctypes.byref(d), ctypes.byref(s), ctypes.byref(p))
        return _device_view_i8(p.value, self.size)

    def writeToDisk(self, path: str) -> None:
        """TemplateVoxelMap::writeToDisk: the reference's binary map file."""
        call("gvx_pvm_write_to_disk", self._h, str(path).encode())

    def readFromDisk(self, path: str) -> None:
        """TemplateVoxelMap::readFromDisk (type and dims must match)."""
        call("gvx_pvm_read_from_disk", self._h, str(path).encode())

    def clearMap(self) -> None:
        call("gvx_pvm_clear", self._h, _stream())

    def insertPointCloud(self, points, meaning: int = eBVM_OCCUPIED, outside: Optional[torch.Tensor] = None) -> None:
        p = _dev_points(points)
        call("gvx_pvm_insert_points", self._h, _ptr(p), p.shape[0], int(meaning), _ptr(outside), _stream())


class BitVectorVoxelMap:
    """BitVoxelMap<256> (GV/voxelmap/BitVoxelMap.h): 32-byte bit vectors."""

    def __init__(self, dims: Sequence[int], voxel_side_length: float):
        self.dims = tuple(int(d) for d in dims)
        self.voxel_side_length = float(voxel_side_length)
        h = ctypes.c_void_p()
        call("gvx_bvm_create", ctypes.byref(Dims(*self.dims)), self.voxel_side_length, ctypes.byref(h))
        self._h = h
        self._destroy = _abi.lib().gvx_bvm_destroy
        self._count = torch.zeros(1, dtype=torch.int64, device="cuda")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            # bound at creation: module globals may already be gone at interpreter exit
            getattr(self, "_destroy", None) and self._destroy(h)
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def size(self) -> int:
        return self.dims[0] * self.dims[1] * self.dims[2]

    def clone(self, other: "BitVectorVoxelMap") -> None:
        """Copy `other`'s bit vectors (equal dims and side length; stream-ordered)."""
        _check_clone(self, other)
        if other is not self:
            self.voxels().copy_(other.voxels())

    def voxels(self) -> torch.Tensor:
        """Borrowed uint8 view of the 32-byte voxels (size * 32 bytes)."""
        d, s, p = Dims(), ctypes.c_float(), ctypes.c_void_p()
        call("gvx_bvm_info", self._h, ctypes.byref(d), ctypes.byref(s), ctypes.byref(p))
        return _device_view_u8(p.value, self.size * 32)

    def writeToDisk(self, path: str) -> None:
        """TemplateVoxelMap::writeToDisk: the reference's binary map file."""
        call("gvx_bvm_write_to_disk", self._h, str(path).encode())

    def readFromDisk(self, path: str) -> None:
        """TemplateVoxelMap::readFromDisk (type and dims must match)."""
        call("gvx_bvm_read_from_disk", self._h, str(path).encode())

    def clearMap(self) -> None:
        call("gvx_bvm_clear", self._h, _stream())

    def insertPointCloud(self, points, meaning: int = eBVM_OCCUPIED, outside: Optional[torch.Tensor] = None) -> None:
        p = _dev_points(points)
        call("gvx_bvm_insert_points", self._h, _ptr(p), p.shape[0], int(meaning), _ptr(outside), _stream())

    def collideWithAsync(self, other, offset=(0, 0, 0), mark: bool = True, out: Optional[torch.Tensor] = None,
                         coll_threshold: float = 1.0) -> torch.Tensor:
        """Stream-ordered collideWith: the count lands in `out` (int64 CUDA)."""
        out = self._count if out is None else out
        if isinstance(other, BitVectorVoxelMap):
            call("gvx_bvm_collide", self._h, other.handle, _offset(offset), 1 if mark else 0, _ptr(out), _stream())
        elif isinstance(other, ProbVoxelMap):
            call("gvx_bvm_collide_pvm", self._h, other.handle, float(coll_threshold), _offset(offset),
                 1 if mark else 0, _ptr(out), _stream())
        else:
            raise TypeError("collideWith expects a BitVectorVoxelMap or a ProbVoxelMap")
        return out

    def collideWith(self, other, coll_threshold: float = 1.0, offset=(0, 0, 0)) -> int:
        """BitVoxelMap::collideWith(BitVectorVoxelMap* | ProbVoxelMap*, coll_threshold, offset):
        the threshold applies to a ProbVoxelMap's occupancy (DefaultCollider)."""
        return int(self.collideWithAsync(other, offset, coll_threshold=coll_threshold).item())

    def collideWithTypes(self, other, coll_threshold: float = 1.0, offset=(0, 0, 0)):
        """-> (count, types uint8[32]): swept-volume types colliding with a
        BitVectorVoxelMap, or this map's types where a ProbVoxelMap is
        occupied; colliding voxels get eBVM_COLLISION.  `offset` is ignored,
        as in the reference."""
        types = torch.zeros(32, dtype=torch.uint8, device="cuda")
        if isinstance(other, BitVectorVoxelMap):
            call("gvx_bvm_collide_types", self._h, other.handle, _ptr(self._count), _ptr(types), _stream())
        elif isinstance(other, ProbVoxelMap):
            call("gvx_bvm_collide_types_pvm", self._h, other.handle, float(coll_threshold), _ptr(self._count),
                 _ptr(types), _stream())
        else:
            raise TypeError("collideWithTypes expects a BitVectorVoxelMap or ProbVoxelMap")
        return int(self._count.item()), types.cpu().numpy()

    def clearBits(self, bits) -> None:
        """BitVoxelMap::clearBits: clear the set bits of `bits` (32 uint8) in every voxel."""
        b = np.ascontiguousarray(np.asarray(bits, dtype=np.uint8).reshape(32))
        call("gvx_bvm_clear_bits", self._h, b.ctypes.data_as(ctypes.c_void_p), _stream())

    def clearBit(self, bit_index: int) -> None:
        b = np.zeros(32, dtype=np.uint8)
        b[int(bit_index) >> 3] = 1 << (int(bit_index) & 7)
        self.clearBits(b)

    def clearBitVoxelMeaning(self, voxel_meaning: int) -> None:
        self.clearBit(voxel_meaning)

    def shiftLeftSweptVolumeIDs(self, shift_size: int) -> None:
        """BitVoxelMap::shiftLeftSweptVolumeIDs: meaning k -> k - shift_size
        (<= 56), meanings 0..3 cleared."""
        call("gvx_bvm_shift_swept_volume_ids", self._h, int(shift_size), _stream())

    def insertMetaPointCloudWithSelfCollisionCheck(self, clouds, meanings=None, masks=None,
                                                   outside: Optional[torch.Tensor] = None):
        """BitVoxelMap::insertMetaPointCloudWithSelfCollisionCheck
        (GV/voxelmap/BitVoxelMap.hpp:227-341).  `clouds`: one (n_k, 3) point set
        per sub-cloud (robot link), inserted in order, each checked against the
        map as the earlier ones left it.  meanings: one meaning per sub-cloud
        (default eBVM_SWEPT_VOLUME_START + k); masks: (n_clouds, 32) uint8 bit
        vectors (default: every bit but eBVM_COLLISION and the own meaning).
        -> (self_collision: bool, colliding meanings uint8[32])."""
        parts = [_dev_points(c) for c in clouds]
        offsets = np.zeros(len(parts) + 1, dtype=np.uint64)
        offsets[1:] = np.cumsum([q.shape[0] for q in parts])
        pts = torch.cat(parts) if parts else torch.zeros((0, 3), dtype=torch.float32, device="cuda")
        mean = None if meanings is None else np.ascontiguousarray(np.asarray(meanings, dtype=np.uint8))
        msk = None if masks is None else np.ascontiguousarray(np.asarray(masks, dtype=np.uint8).reshape(len(parts), 32))
        colliding = np.zeros(32, dtype=np.uint8)
        anyc = ctypes.c_int(0)
        call("gvx_bvm_insert_meta_points_self_coll", self._h, _ptr(pts),
             offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), len(parts),
             None if mean is None else mean.ctypes.data_as(ctypes.c_void_p),
             None if msk is None else msk.ctypes.data_as(ctypes.c_void_p),
             colliding.ctypes.data_as(ctypes.c_void_p), ctypes.byref(anyc), _ptr(outside), _stream())
        return bool(anyc.value), colliding


class BitVectorVoxelList:
    """BitVoxelList<256, uint32> (GV/voxellist/BitVoxelList.h): sorted unique
    voxel ids with 32-byte bit vectors, tied to a reference map's dims."""

    def __init__(self, ref_dims: Sequence[int], voxel_side_length: float):
        self.dims = tuple(int(d) for d in ref_dims)
        self.voxel_side_length = float(voxel_side_length)
        h = ctypes.c_void_p()
        call("gvx_blist_create", ctypes.byref(Dims(*self.dims)), self.voxel_side_length, ctypes.byref(h))
        self._h = h
        self._destroy = _abi.lib().gvx_blist_destroy
        self._count = torch.zeros(1, dtype=torch.int64, device="cuda")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            # bound at creation: module globals may already be gone at interpreter exit
            getattr(self, "_destroy", None) and self._destroy(h)
            self._h = None

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def getDimensions(self) -> int:
        n = ctypes.c_uint64()
        call("gvx_blist_size", self._h, ctypes.byref(n))
        return n.value

    def shiftLeftSweptVolumeIDs(self, shift_size: int) -> None:
        """BitVoxelList::shiftLeftSweptVolumeIDs: meaning k -> k - shift_size (<= 56)
        in every entry, meanings 0..3 cleared."""
        call("gvx_blist_shift_swept_volume_ids", self._h, int(shift_size), _stream())

    def clearBitVoxelMeaning(self, voxel_meaning: int) -> None:
        b = np.zeros(32, dtype=np.uint8)
        b[int(voxel_meaning) >> 3] = 1 << (int(voxel_meaning) & 7)
        call("gvx_blist_clear_bits", self._h, b.ctypes.data_as(ctypes.c_void_p), _stream())

    def ids(self) -> torch.Tensor:
        n = self.getDimensions()
        pi, pv = ctypes.c_void_p(), ctypes.c_void_p()
        call("gvx_blist_data", self._h, ctypes.byref(pi), ctypes.byref(pv))
        return _device_view(pi.value, n).clone() if n else torch.empty(0, dtype=torch.int32, device="cuda")

    def voxels(self) -> torch.Tensor:
        n = self.getDimensions()
        pi, pv = ctypes.c_void_p(), ctypes.c_void_p()
        call("gvx_blist_data", self._h, ctypes.byref(pi), ctypes.byref(pv))
        return _device_view_u8(pv.value, n * 32).clone() if n else torch.empty(0, dtype=torch.uint8, device="cuda")

    def clearMap(self) -> None:
        call("gvx_blist_clear", self._h)

    def insertPointCloud(self, points, meaning: int = eBVM_OCCUPIED) -> None:
        p = _dev_points(points)
        call("gvx_blist_insert_points", self._h, _ptr(p), p.shape[0], int(meaning), _stream())

    def set(self, ids: torch.Tensor, voxels: Optional[torch.Tensor] = None, meaning: int = eBVM_OCCUPIED) -> None:
        ids = _dev_u32(ids)
        call("gvx_blist_set", self._h, _ptr(ids), _ptr(voxels), ids.shape[0], int(meaning), _stream())

    def collideWith(self, other, coll_threshold: float = 1.0, offset=(0, 0, 0), mark: bool = True) -> int:
        if isinstance(other, BitVectorVoxelMap):
            call("gvx_blist_collide_bvm", self._h, other.handle, _offset(offset), 1 if mark else 0, _ptr(self._count),
                 _stream())
        elif isinstance(other, ProbVoxelMap):
            call("gvx_blist_collide_pvm", self._h, other.handle, float(coll_threshold), _offset(offset),
                 1 if mark else 0, _ptr(self._count), _stream())
        elif isinstance(other, BitVectorVoxelList):
            call("gvx_blist_collide_blist", self._h, other.handle, _offset(offset), _ptr(self._count), _stream())
        else:
            raise TypeError("collideWith expects a BitVectorVoxelMap, ProbVoxelMap or BitVectorVoxelList")
        return int(self._count.item())

    def collideWithTypes(self, other, coll_threshold: float = 1.0, offset=(0, 0, 0)):
        """-> (count, types uint8[32]) against a BitVectorVoxelMap, a ProbVoxelMap
        or another BitVectorVoxelList; colliding entries get eBVM_COLLISION
        (not for list vs list)."""
        types = torch.zeros(32, dtype=torch.uint8, device="cuda")
        if isinstance(other, BitVectorVoxelMap):
            call("gvx_blist_collide_types_bvm", self._h, other.handle, _offset(offset), _ptr(self._count), _ptr(types),
                 _stream())
        elif isinstance(other, ProbVoxelMap):
            call("gvx_blist_collide_types_pvm", self._h, other.handle, float(coll_threshold), _offset(offset),
                 _ptr(self._count), _ptr(types), _stream())
        elif isinstance(other, BitVectorVoxelList):
            call("gvx_blist_collide_types_blist", self._h, other.handle, _ptr(self._count), _ptr(types), _stream())
        else:
            raise TypeError("collideWithTypes expects a BitVectorVoxelMap, ProbVoxelMap or BitVectorVoxelList")
        return int(self._count.item()), types.cpu().numpy()

    def collideWithTypeMask(self, other: "BitVectorVoxelMap", types_to_check, coll_threshold: float = 1.0,
                            offset=(0, 0, 0)) -> int:
        """Collisions of entries whose bits meet the 32-byte mask."""
        mask = torch.as_tensor(np.asarray(types_to_check, dtype=np.uint8)).cuda()
        call("gvx_blist_collide_type_mask_bvm", self._h, other.handle, _ptr(mask), _offset(offset), _ptr(self._count),
             _stream())
        return int(self._count.item())


def set_query_config(threads: int = 256, blocks_per_sm: int = 16) -> None:
    """Fix the launch shape of the trilinear query kernels (threads 64, 128,
    256 or 512; blocks_per_sm 1..64).  Results do not depend on it."""
    c = _abi.QueryConfig(threads, blocks_per_sm, 0.0)
    call("gvx_set_query_config", ctypes.byref(c))


def lists_collide_map(ids: torch.Tensor, voxels: torch.Tensor, offsets: torch.Tensor, bvm: BitVectorVoxelMap,
                      mark: bool = False, counts: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Batched list-vs-map collision: CSR lists, one launch, per-list counts."""
    n_lists = offsets.shape[0] - 1
    counts = torch.empty(n_lists, dtype=torch.int64, device="cuda") if counts is None else counts
    call("gvx_lists_collide_bvm", _ptr(ids), _ptr(voxels), _ptr(offsets), n_lists, ids.shape[0], bvm.handle,
         1 if mark else 0, _ptr(counts), _stream())
    return counts


def make_arm(spec: dict) -> Arm:
    """Pack an arm description (dict of lists) into the C struct."""
    arm = Arm()
    arm.n_joints = int(spec["n_joints"])
    arm.n_spheres = int(len(spec["r"]))
    for i, v in enumerate(spec["base"]):
        arm.base[i] = float(v)
    for j in range(arm.n_joints):
        arm.theta[j] = float(spec["theta"][j])
        arm.d[j] = float(spec["d"][j])
        arm.a[j] = float(spec["a"][j])
        arm.alpha[j] = float(spec["alpha"][j])
    for s in range(arm.n_spheres):
        arm.link[s] = int(spec["link"][s])
        arm.t[s] = float(spec["t"][s])
        arm.r[s] = float(spec["r"][s])
    return arm
