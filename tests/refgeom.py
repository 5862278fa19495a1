"""Geometry generators of gpu-voxels' test suite, restated in numpy float32
(GV = packages/gpu_voxels/src/gpu_voxels/):
  createEquidistantPointsInBox        GV/helpers/GeometryGeneration.cpp:237-264
  createNonOverlapping3dCheckerboard  GV/helpers/GeometryGeneration.cpp:266-297
  createBoxOfPoints                   GV/helpers/GeometryGeneration.cpp:90-107
The loops keep the reference's float32 accumulation so the same voxels are hit.
"""
from __future__ import annotations

import numpy as np


def equidistant_points_in_box(max_points: int, dims, side: float) -> np.ndarray:
    out = []
    s = np.float32(side)
    for i in range((dims[0] - 1) // 2):
        for j in range((dims[1] - 1) // 2):
            for k in range((dims[2] - 1) // 2):
                if len(out) >= max_points:
                    return np.asarray(out, dtype=np.float32).reshape(-1, 3)
                out.append((np.float32(i * 2 * s + s / 2.0), np.float32(j * 2 * s + s / 2.0),
                            np.float32(k * 2 * s + s / 2.0)))
    return np.asarray(out, dtype=np.float32).reshape(-1, 3)


def equidistant_points_fast(max_points: int, dims, side: float) -> np.ndarray:
    """Vectorised form of equidistant_points_in_box (same order and values)."""
    ni, nj, nk = ((d - 1) // 2 for d in dims)
    i, j, k = np.meshgrid(np.arange(ni), np.arange(nj), np.arange(nk), indexing="ij")
    s = np.float64(np.float32(side))
    pts = np.stack([i.ravel() * 2 * s + s / 2.0, j.ravel() * 2 * s + s / 2.0, k.ravel() * 2 * s + s / 2.0], axis=1)
    return pts[:max_points].astype(np.float32)


def nonoverlapping_checkerboard(max_points: int, dims, side: float):
    ni, nj, nk = ((d - 1) // 2 for d in dims)
    i, j, k = np.meshgrid(np.arange(ni), np.arange(nj), np.arange(nk), indexing="ij")
    s = np.float64(np.float32(side))
    i, j, k = i.ravel()[:max_points], j.ravel()[:max_points], k.ravel()[:max_points]
    black = np.stack([i * 2 * s + s / 2.0, j * 2 * s + s / 2.0, k * 2 * s + s / 2.0], axis=1).astype(np.float32)
    white = np.stack([(i * 2 + 1) * s + s / 2.0, (j * 2 + 1) * s + s / 2.0, (k * 2 + 1) * s + s / 2.0],
                     axis=1).astype(np.float32)
    return black, white


def _frange(lo, hi, delta):
    v = np.float32(lo)
    d = np.float32(delta)
    out = []
    while v <= np.float32(hi):
        out.append(v)
        v = np.float32(v + d)
    return out


def box_of_points(lo, hi, delta) -> np.ndarray:
    xs, ys, zs = (_frange(lo[a], hi[a], delta) for a in range(3))
    pts = [(x, y, z) for x in xs for y in ys for z in zs]
    return np.asarray(pts, dtype=np.float32).reshape(-1, 3)
