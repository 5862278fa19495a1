"""Points on voxel faces: coordinates k * s (formed in float32, as a caller's
float pose arithmetic would) and their float neighbours one ulp either side,
for side lengths that are and are not exact in binary, including the upper
map face k = dim (outside).  The voxel is floor(c / s) with an IEEE float32
divide (mapToVoxels, GV/voxelmap/kernels/VoxelMapOperations.h:121-131), so a
point one ulp below k * s may land in voxel k - 1 and k * s itself in k or
k - 1 depending on the rounding of the quotient; every insert path must agree
with the oracle on each of them."""
import numpy as np
import pytest
import torch

import gvx
import oracle
from gpu_helpers import oracle_edt, to_u32
from gvx.batch import Batch

DIMS = (37, 29, 23)
SIDES = (0.01, 0.005, 0.03, 0.1, 0.25, 1.0)


def face_points(dims, side, n=20_000, seed=0):
    rng = np.random.default_rng(seed)
    s = np.float32(side)
    axes = []
    for d in dims:
        k = np.arange(d + 1, dtype=np.float32)
        c = k * s
        axes.append(np.concatenate([c, np.nextafter(c, np.float32(np.inf)), np.nextafter(c, np.float32(-np.inf)),
                                    (np.arange(d + 1, dtype=np.float64) * side).astype(np.float32)]))
    pts = np.stack([rng.choice(a, n) for a in axes], axis=1).astype(np.float32)
    return pts


def test_oracle_voxel_of_face_points_is_the_float32_quotient():
    """The oracle's voxel index equals floor(float32(c) / float32(s)) computed by numpy."""
    for side in SIDES:
        pts = face_points(DIMS, side, 3000, 1)
        want = np.floor(pts / np.float32(side)).astype(np.int64)
        got = np.array([[oracle.coord_to_voxel(float(c), side) for c in p] for p in pts[:400]])
        assert np.array_equal(got, np.maximum(want[:400], 0)), side


@pytest.mark.gpu
@pytest.mark.parametrize("side", SIDES)
def test_face_points_every_insert_path(side):
    pts = face_points(DIMS, side, seed=int(side * 1000))
    p = torch.as_tensor(pts).cuda()
    ins_o, edt_o = oracle_edt(DIMS, side, pts)
    out_o = oracle.dvm_insert(oracle.dvm_empty(DIMS), DIMS, side, pts)
    assert out_o  # the k = dim face is outside

    m = gvx.DistanceVoxelMap(DIMS, side)
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    m.insertPointCloud(p, outside=flag)
    assert np.array_equal(to_u32(m.data()), ins_o)
    assert bool(flag.item()) == out_o
    m.parallelBanding3D()
    assert np.array_equal(to_u32(m.data()), edt_o)

    flag.zero_()
    m.voxelize_edt(p, outside=flag)
    assert np.array_equal(to_u32(m.data()), edt_o)
    assert bool(flag.item()) == out_o

    b = gvx.BitVectorVoxelMap(DIMS, side)
    flag.zero_()
    b.insertPointCloud(p, 7, outside=flag)
    want_b = oracle.bvm_empty(DIMS)
    assert oracle.bvm_insert(want_b, DIMS, side, pts, 7) == bool(flag.item())
    assert np.array_equal(b.voxels().cpu().numpy().reshape(-1), want_b.reshape(-1))

    pm = gvx.ProbVoxelMap(DIMS, side)
    flag.zero_()
    pm.insertPointCloud(p, outside=flag)
    want_p = oracle.pvm_empty(DIMS)
    assert oracle.pvm_insert(want_p, DIMS, side, pts, gvx.eBVM_OCCUPIED) == bool(flag.item())
    assert np.array_equal(pm.data().cpu().numpy().reshape(-1), want_p.reshape(-1))

    maps = [gvx.DistanceVoxelMap(DIMS, side), gvx.DistanceVoxelMap(DIMS, side)]
    bt = Batch(maps)
    half = pts.shape[0] // 2
    offs = torch.tensor([0, half, pts.shape[0]], dtype=torch.int64, device="cuda")
    bt.voxelize_edt(p, offs)
    assert bt.edt_check() == 0
    for k, (a, e) in enumerate(((0, half), (half, pts.shape[0]))):
        _, want = oracle_edt(DIMS, side, pts[a:e])
        assert np.array_equal(to_u32(maps[k].data()), want), k
