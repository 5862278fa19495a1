"""ProbVoxelMap insert and DistanceVoxelMap.mergeOccupied on the GPU against
the oracle, bit for bit, including many points per voxel (every update is
applied), all meanings, offsets and the EDT of the merged map."""
import numpy as np
import pytest
import torch

import gvx
import oracle
import refgeom
from gpu_helpers import to_u32

pytestmark = pytest.mark.gpu


def _pvm_both(dims, side, batches):
    g = gvx.ProbVoxelMap(dims, side)
    o = oracle.pvm_empty(dims)
    for pts, meaning in batches:
        flag = torch.zeros(1, dtype=torch.int32, device="cuda")
        g.insertPointCloud(torch.as_tensor(pts).cuda(), meaning, outside=flag)
        want_flag = oracle.pvm_insert(o, dims, side, pts, meaning)
        assert bool(flag.item()) == want_flag
    return g, o


def test_pvm_insert_all_meanings_and_duplicates():
    dims = (37, 29, 23)
    rng = np.random.default_rng(0)
    batches = []
    for meaning in [1, 1, 0, 254, 4, 2, 129, 3, 77, 255, 1]:
        n = int(rng.integers(50, 4000))
        pts = (rng.random((n, 3)) * np.asarray(dims) * 1.1 - 0.5).astype(np.float32)  # some outside
        pts[: n // 3] = pts[0]  # a third of the points share one voxel
        batches.append((pts, meaning))
    g, o = _pvm_both(dims, 1.0, batches)
    assert np.array_equal(g.data().cpu().numpy(), o)


def test_merge_occupied_example_and_edt():
    dims = (128, 128, 128)
    box1 = refgeom.box_of_points((40, 40, 40), (60, 60, 60), 0.9)
    box2 = refgeom.box_of_points((50, 50, 50), (70, 70, 70), 0.9)
    g, o = _pvm_both(dims, 1.0, [(box1, 254), (box2, 4)])
    assert np.array_equal(g.data().cpu().numpy(), o)
    for off, thr in [((0, 0, 0), 0.55), ((3, 1, 2), 0.55), ((0, 0, 0), 0.0), ((5, 0, 0), 1.0)]:
        d = gvx.DistanceVoxelMap(dims, 1.0)
        d.mergeOccupied(g, off, thr)
        want = oracle.dvm_empty(dims)
        oracle.dvm_merge_occupied(want, o, dims, off, thr)
        assert np.array_equal(to_u32(d.data()), want), (off, thr)
    d = gvx.DistanceVoxelMap(dims, 1.0)
    d.mergeOccupied(g, (0, 0, 0), 0.55)
    assert int((d.data() != 0x3FFFFFFF).sum().item()) == 20 ** 3 - 10 ** 3
    d.parallelBanding3D()
    want = oracle.dvm_empty(dims)
    oracle.dvm_merge_occupied(want, o, dims, (0, 0, 0), 0.55)
    oracle.pba(want, dims)
    assert np.array_equal(to_u32(d.data()), want)


def test_merge_keeps_existing_sites_and_rejects_other_dims():
    dims = (40, 33, 21)
    rng = np.random.default_rng(3)
    g, o = _pvm_both(dims, 0.5, [((rng.random((3000, 3)) * np.asarray(dims) * 0.5).astype(np.float32), 1)])
    d = gvx.DistanceVoxelMap(dims, 0.5)
    pts = (rng.random((500, 3)) * np.asarray(dims) * 0.5).astype(np.float32)
    d.insertPointCloud(torch.as_tensor(pts).cuda())
    want = oracle.dvm_empty(dims)
    oracle.dvm_insert(want, dims, 0.5, pts)
    d.mergeOccupied(g, (0, 0, 0), 0.6)
    oracle.dvm_merge_occupied(want, o, dims, (0, 0, 0), 0.6)
    assert np.array_equal(to_u32(d.data()), want)
    with pytest.raises(gvx.GvxError):
        gvx.DistanceVoxelMap((40, 33, 22), 0.5).mergeOccupied(g)
