"""Batched processing of many DistanceVoxelMaps (gvx_batch_* in include/gvx.h).

    b = Batch([map0, map1, ...])
    b.clear(); b.insert(points_cat, offsets); b.edt(); d, g = b.query(q_xyz, q_map)
    b.capture(points_cat, offsets, q_xyz, q_map)   # record the step as a CUDA graph
    b.replay()                                     # one launch call per step
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import torch

from ._abi import call, lib
from .maps import DistanceVoxelMap, _ptr, _stream


class Batch:
    def __init__(self, maps: Sequence[DistanceVoxelMap]):
        self.maps = list(maps)  # keep the maps alive as long as the batch
        arr = (ctypes.c_void_p * len(self.maps))(*[m.handle.value for m in self.maps])
        h = ctypes.c_void_p()
        call("gvx_batch_create", arr, len(self.maps), ctypes.byref(h))
        self._h = h
        self._destroy = lib().gvx_batch_destroy  # bound now: module globals may be gone at exit
        self._graph_bufs = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            getattr(self, "_destroy", None) and self._destroy(h)
            self._h = None

    def clear(self) -> None:
        call("gvx_batch_clear", self._h, _stream())

    def insert(self, xyz: torch.Tensor, offsets: torch.Tensor) -> None:
        """xyz: [N,3] float32 CUDA; offsets: int64 CUDA [n_maps+1] (map k owns offsets[k]..offsets[k+1])."""
        call("gvx_batch_insert_points", self._h, _ptr(xyz), _ptr(offsets), xyz.shape[0], _stream())

    def edt(self) -> None:
        call("gvx_batch_edt", self._h, _stream())

    def voxelize_edt(self, xyz: torch.Tensor, offsets: torch.Tensor) -> None:
        """clear + insert + edt in one call (same result)."""
        call("gvx_batch_voxelize_edt", self._h, _ptr(xyz), _ptr(offsets), xyz.shape[0], _stream())

    def autotune(self, force: bool = False) -> dict:
        """Pick the fastest sweep configuration of the batched EDT (the maps'
        content is saved and restored around the timing runs)."""
        from ._abi import EdtConfig
        c = EdtConfig()
        call("gvx_batch_autotune", self._h, int(bool(force)), ctypes.byref(c), _stream())
        return {"rows": c.rows, "fused": c.fused, "ms": c.ms}

    def edt_check(self) -> int:
        """Synchronise and return the error word of the last batched EDT (0 = ok)."""
        flags = ctypes.c_uint32(0)
        call("gvx_batch_edt_check", self._h, ctypes.byref(flags))
        return int(flags.value)

    def query(self, xyz: torch.Tensor, map_index: torch.Tensor, with_grad: bool = True):
        n = xyz.shape[0]
        dist = torch.empty(n, dtype=torch.float32, device="cuda")
        grad = torch.empty(n, 3, dtype=torch.float32, device="cuda") if with_grad else None
        call("gvx_batch_query_trilinear", self._h, _ptr(xyz), _ptr(map_index), n, _ptr(dist), _ptr(grad), _stream())
        return (dist, grad) if with_grad else dist

    def capture(self, xyz: torch.Tensor, offsets: torch.Tensor, q_xyz: torch.Tensor, q_map: torch.Tensor):
        """Record clear -> insert -> EDT -> queries on these buffers as one CUDA graph.
        Returns the (dist, grad) output tensors the graph writes."""
        n_q = q_xyz.shape[0]
        dist = torch.empty(n_q, dtype=torch.float32, device="cuda")
        grad = torch.empty(n_q, 3, dtype=torch.float32, device="cuda")
        self._graph_bufs = (xyz, offsets, q_xyz, q_map, dist, grad)
        call("gvx_batch_graph_capture", self._h, _ptr(xyz), _ptr(offsets), xyz.shape[0], _ptr(q_xyz), _ptr(q_map), n_q,
             _ptr(dist), _ptr(grad), _stream())
        return dist, grad

    def replay(self) -> None:
        call("gvx_batch_graph_launch", self._h, _stream())
