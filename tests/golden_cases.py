"""Seeded input cases of the golden fixtures (tests/golden/ref_*.npz), inside
the reference's PBA domain (x == y, x % 64 == 0)."""
import numpy as np

import refgeom

CASES = {
    "random64": {"dims": (64, 64, 64), "side": 1.0, "kind": "uniform", "n": 400, "seed": 0},
    "lattice64x40": {"dims": (64, 64, 40), "side": 1.0, "kind": "lattice", "n": 100_000},
    "dense64": {"dims": (64, 64, 64), "side": 1.0, "kind": "uniform", "n": 60_000, "seed": 1},
    "symmetric": {"dims": (64, 64, 64), "side": 1.0, "kind": "fixed",
                  "pts": [[10.5, 32.5, 20.5], [53.5, 32.5, 20.5]]},
    "negative_and_outside": {"dims": (64, 64, 32), "side": 0.5, "kind": "uniform_wide", "n": 2000, "seed": 2},
    "boxes128x20": {"dims": (128, 128, 20), "side": 0.01, "kind": "boxes", "seed": 3},
}


def points_for(spec) -> np.ndarray:
    dims = np.asarray(spec["dims"], dtype=np.float64)
    side = spec["side"]
    kind = spec["kind"]
    if kind == "uniform":
        rng = np.random.default_rng(spec["seed"])
        return (rng.random((spec["n"], 3)) * dims * side).astype(np.float32)
    if kind == "uniform_wide":
        rng = np.random.default_rng(spec["seed"])
        return ((rng.random((spec["n"], 3)) * 1.4 - 0.2) * dims * side).astype(np.float32)
    if kind == "lattice":
        return refgeom.equidistant_points_fast(spec["n"], spec["dims"], side)
    if kind == "fixed":
        return np.asarray(spec["pts"], dtype=np.float32)
    if kind == "boxes":
        import workloads
        return workloads.box_scene(spec["seed"], dims * side, n_boxes=12, n_points=20_000)
    raise ValueError(kind)


# Lists of voxel ids against one BitVectorVoxelMap (the reference's
# kernelCollideWithVoxelMap, GV/voxellist/kernels/VoxelListOperations.hpp:146-197).
# The map holds occupied voxels and free-only voxels (which never collide);
# the lists hold random sorted unique ids -- a few beyond the map -- with a
# meaning of their own, some entries free-only.
LIST_CASE = {"dims": (64, 48, 40), "map_seed": 21, "map_points": 15_000, "free_points": 5_000, "n_lists": 12,
             "min_len": 50, "max_len": 3_000, "seed": 22, "offsets": [(0, 0, 0), (1, 0, 0), (-3, 2, 1), (0, 0, 5)]}


def list_inputs(spec=LIST_CASE):
    """-> (bvm uint8[n*32], ids uint32, list voxels uint8[len(ids)*32], offsets uint64[n_lists+1])."""
    import oracle

    dims = spec["dims"]
    nvox = int(np.prod(dims))
    rng = np.random.default_rng(spec["map_seed"])
    bmap = oracle.bvm_empty(dims)
    oracle.bvm_insert(bmap, dims, 1.0, (rng.random((spec["map_points"], 3)) * dims).astype(np.float32), 1)
    oracle.bvm_insert(bmap, dims, 1.0, (rng.random((spec["free_points"], 3)) * dims).astype(np.float32), 0)
    rng = np.random.default_rng(spec["seed"])
    ids, vox, offs = [], [], [0]
    for k in range(spec["n_lists"]):
        n = int(rng.integers(spec["min_len"], spec["max_len"]))
        v = np.unique(rng.integers(0, nvox + 64, size=n)).astype(np.uint32)
        bits = np.zeros((v.shape[0], 32), dtype=np.uint8)
        meaning = 4 + k
        bits[:, meaning >> 3] |= np.uint8(1 << (meaning & 7))
        free_only = rng.random(v.shape[0]) < 0.1
        bits[free_only] = 0
        bits[free_only, 0] = 1
        ids.append(v)
        vox.append(bits.reshape(-1))
        offs.append(offs[-1] + v.shape[0])
    return bmap, np.concatenate(ids), np.concatenate(vox), np.asarray(offs, dtype=np.uint64)


def linear_offset(dims, off) -> int:
    """getVoxelIndexSigned (GV/voxelmap/kernels/VoxelMapOperations.h): z*X*Y + y*X + x."""
    return int(off[2]) * dims[0] * dims[1] + int(off[1]) * dims[0] + int(off[0])
