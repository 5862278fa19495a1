"""Batched maps of uneven dims: one launch per step over all maps (and the
CUDA-graph replay of the whole step) gives exactly the per-map results."""
import numpy as np
import pytest
import torch

import gvx
import oracle
import workloads
from gvx.batch import Batch
from gpu_helpers import to_u32

pytestmark = pytest.mark.gpu


def _scenes(n=6, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        dims = tuple(int(v) for v in rng.integers(20, 140, size=3))
        side = 0.01
        pts = workloads.box_scene(200 + i, np.asarray(dims) * side, n_boxes=6, n_points=int(rng.integers(500, 20000)))
        out.append((dims, side, pts))
    return out


def _cat(scenes):
    pts = np.concatenate([p for _, _, p in scenes]).astype(np.float32)
    offs = np.zeros(len(scenes) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([p.shape[0] for _, _, p in scenes])
    return torch.as_tensor(pts).cuda(), torch.as_tensor(offs).cuda()


def _queries(scenes, per_map=500, seed=9):
    rng = np.random.default_rng(seed)
    q, mi = [], []
    for k, (dims, side, _) in enumerate(scenes):
        q.append(((0.5 + rng.random((per_map, 3)) * (np.asarray(dims) - 1)) * side).astype(np.float32))
        mi.append(np.full(per_map, k, dtype=np.int32))
    return torch.as_tensor(np.concatenate(q)).cuda(), torch.as_tensor(np.concatenate(mi)).cuda()


def test_batch_edt_equals_per_map_and_oracle():
    scenes = _scenes()
    maps = [gvx.DistanceVoxelMap(d, s) for d, s, _ in scenes]
    b = Batch(maps)
    pts, offs = _cat(scenes)
    b.clear()
    b.insert(pts, offs)
    b.edt()
    q, qm = _queries(scenes)
    dist, grad = b.query(q, qm)
    assert b.edt_check() == 0
    for k, (dims, side, p) in enumerate(scenes):
        want = oracle.dvm_empty(dims)
        oracle.dvm_insert(want, dims, side, p)
        oracle.pba(want, dims)
        assert np.array_equal(to_u32(maps[k].data()), want), f"map {k} {dims}"
        sel = (qm == k)
        d1, g1 = maps[k].trilinear(q[sel])
        assert torch.equal(dist[sel], d1) and torch.equal(grad[sel], g1)


def test_batch_graph_replay_matches_eager():
    scenes = _scenes(5, seed=7)
    maps = [gvx.DistanceVoxelMap(d, s) for d, s, _ in scenes]
    b = Batch(maps)
    pts, offs = _cat(scenes)
    q, qm = _queries(scenes, 300, seed=3)
    b.clear(); b.insert(pts, offs); b.edt()
    d_eager, g_eager = b.query(q, qm)
    eager_maps = [to_u32(m.data()) for m in maps]
    dist, grad = b.capture(pts, offs, q, qm)
    for m in maps:
        m.clearMap()
    for _ in range(3):
        b.replay()
    torch.cuda.synchronize()
    for k in range(len(maps)):
        assert np.array_equal(to_u32(maps[k].data()), eager_maps[k])
    assert torch.equal(dist, d_eager) and torch.equal(grad, g_eager)


def test_batch_voxelize_edt_equals_clear_insert_edt():
    scenes = _scenes(6, seed=11)
    maps_a = [gvx.DistanceVoxelMap(d, s) for d, s, _ in scenes]
    maps_b = [gvx.DistanceVoxelMap(d, s) for d, s, _ in scenes]
    pts, offs = _cat(scenes)
    a, b = Batch(maps_a), Batch(maps_b)
    a.clear(); a.insert(pts, offs); a.edt()
    b.voxelize_edt(pts, offs)
    assert b.edt_check() == 0
    for ma, mb in zip(maps_a, maps_b):
        assert torch.equal(ma.data(), mb.data())


def test_batch_thin_maps_items_span_slices():
    """Maps with x or y below 32 (or 1): one warp item covers columns of several
    z slices, so Y items bump and X items wait on several slice counters."""
    dims_list = [(1, 40, 60), (5, 3, 100), (33, 1, 20), (70, 9, 2), (1, 1, 300), (31, 33, 17)]
    rng = np.random.default_rng(21)
    scenes = []
    for dims in dims_list:
        n = max(1, int(np.prod(dims)) // 50)
        pts = (rng.random((n, 3)) * np.asarray(dims)).astype(np.float32)
        scenes.append((dims, 1.0, pts))
    maps = [gvx.DistanceVoxelMap(d, s) for d, s, _ in scenes]
    b = Batch(maps)
    pts, offs = _cat(scenes)
    b.voxelize_edt(pts, offs)
    assert b.edt_check() == 0
    got_fused = [to_u32(m.data()).copy() for m in maps]
    b.clear()
    b.insert(pts, offs)
    b.edt()
    assert b.edt_check() == 0
    for k, (dims, side, p) in enumerate(scenes):
        want = oracle.dvm_empty(dims)
        oracle.dvm_insert(want, dims, side, p)
        oracle.pba(want, dims)
        assert np.array_equal(got_fused[k], want), f"voxelize_edt map {k} {dims}"
        assert np.array_equal(to_u32(maps[k].data()), want), f"edt map {k} {dims}"


def test_batch_edt_per_map_route_own_and_other_sites():
    """Batch.edt on filled maps picks pass Z's route per map: the occupancy-bit
    pass when every voxel is UNINIT or its own site, the general pass
    otherwise (each launch skips the other maps).  A batch mixing freshly
    inserted maps with maps that still hold an earlier transform (every voxel
    its nearest site) equals the oracle map by map, and so does a second EDT
    of the whole batch, where every map holds other sites."""
    scenes = _scenes(6, seed=13)
    maps = [gvx.DistanceVoxelMap(d, s) for d, s, _ in scenes]
    b = Batch(maps)
    pts, offs = _cat(scenes)
    b.clear()
    b.insert(pts, offs)
    b.edt()
    for k in range(0, len(maps), 2):  # even maps back to their inserted state
        maps[k].clearMap()
        maps[k].insertPointCloud(torch.as_tensor(scenes[k][2].astype(np.float32)).cuda())
    for rep in range(2):
        inputs = [to_u32(m.data()).copy() for m in maps]
        b.edt()
        assert b.edt_check() == 0
        for k, (dims, _, _) in enumerate(scenes):
            want = inputs[k].copy()
            oracle.pba(want, dims)
            assert np.array_equal(to_u32(maps[k].data()), want), f"pass {rep} map {k} {dims}"
