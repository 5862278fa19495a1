"""The EDT autotuner: every configuration it chooses between gives the same
map bit for bit, tuning leaves the map's content alone, and its choice is
cached in memory and, through GVX_TUNE_CACHE, across processes."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

import gvx
import oracle
from gpu_helpers import to_u32
import workloads
from gvx.batch import Batch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _scene(dims, seed, n=3000):
    return workloads.box_scene(seed, np.asarray(dims) * 0.01, n_boxes=8, n_points=n).astype(np.float32)


def test_every_config_is_bit_identical_and_tuning_keeps_the_map():
    dims = (96, 80, 64)
    pts = _scene(dims, 1)
    want = oracle.dvm_empty(dims)
    oracle.dvm_insert(want, dims, 0.01, pts)
    oracle.pba(want, dims)
    m = gvx.DistanceVoxelMap(dims, 0.01)
    for rows in (16, 32):
        for fused in (0, 1):
            m.clearMap()
            m.insertPointCloud(torch.as_tensor(pts).cuda())
            m.set_edt_config(rows, fused)
            m.parallelBanding3D()
            assert m.edt_check() == 0
            assert np.array_equal(to_u32(m.data()), want), (rows, fused)
    m.clearMap()
    m.insertPointCloud(torch.as_tensor(pts).cuda())
    before = m.data().clone()
    cfg = m.autotune(force=True)
    assert cfg["rows"] in (16, 32) and cfg["fused"] in (0, 1) and cfg["ms"] > 0
    assert torch.equal(m.data(), before)  # tuning ran on a copy
    again = m.autotune()  # cached: same choice, same recorded time
    assert again == cfg
    m.parallelBanding3D()
    assert np.array_equal(to_u32(m.data()), want)


def test_tune_cache_file_is_shared_between_processes(tmp_path):
    cache = tmp_path / "gvx_tune.txt"
    script = textwrap.dedent(f"""
        import sys, json
        sys.path.insert(0, {os.path.join(ROOT, 'gpu-voxels_b200')!r})
        import numpy as np, torch, gvx
        m = gvx.DistanceVoxelMap((64, 48, 40), 0.01)
        m.insertPointCloud(torch.rand(2000, 3, device='cuda') * torch.tensor([0.64, 0.48, 0.40], device='cuda'))
        print(json.dumps(m.autotune()))
    """)
    env = dict(os.environ, GVX_TUNE_CACHE=str(cache))
    outs = [subprocess.run([sys.executable, "-c", script], env=env, capture_output=True, text=True, timeout=300)
            for _ in range(2)]
    for o in outs:
        assert o.returncode == 0, o.stderr[-2000:]
    first, second = [o.stdout.strip().splitlines()[-1] for o in outs]
    assert first == second  # the second process took the first one's entry
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and "|map|64x48x40" in lines[0]


def test_batch_autotune_restores_maps_and_stays_exact():
    rng = np.random.default_rng(4)
    scenes = []
    for i in range(5):
        dims = tuple(int(v) for v in rng.integers(30, 120, size=3))
        scenes.append((dims, _scene(dims, 30 + i, 2000)))
    maps = [gvx.DistanceVoxelMap(d, 0.01) for d, _ in scenes]
    b = Batch(maps)
    pts = torch.as_tensor(np.concatenate([p for _, p in scenes])).cuda()
    offs = torch.as_tensor(np.concatenate([[0], np.cumsum([p.shape[0] for _, p in scenes])]).astype(np.int64)).cuda()
    b.clear()
    b.insert(pts, offs)
    before = [m.data().clone() for m in maps]
    cfg = b.autotune(force=True)
    assert cfg["rows"] in (16, 32) and cfg["fused"] == 1
    for m, w in zip(maps, before):
        assert torch.equal(m.data(), w)
    b.edt()
    assert b.edt_check() == 0
    for k, (dims, p) in enumerate(scenes):
        want = oracle.dvm_empty(dims)
        oracle.dvm_insert(want, dims, 0.01, p)
        oracle.pba(want, dims)
        assert np.array_equal(to_u32(maps[k].data()), want), dims


def test_query_launch_shapes_are_bit_identical_and_autotune_picks_one():
    dims = (90, 70, 50)
    pts = _scene(dims, 7)
    m = gvx.DistanceVoxelMap(dims, 0.01)
    m.insertPointCloud(torch.as_tensor(pts).cuda())
    m.parallelBanding3D()
    rng = np.random.default_rng(3)
    q = torch.as_tensor(((0.5 + rng.random((70_001, 3)) * (np.asarray(dims) - 1)) * 0.01).astype(np.float32)).cuda()
    up = torch.as_tensor(rng.standard_normal(q.shape[0]).astype(np.float32)).cuda()
    b = Batch([m])
    mi = torch.zeros(q.shape[0], dtype=torch.int32, device="cuda")
    gvx.set_query_config(256, 16)
    d0, g0 = m.trilinear(q)
    a0 = m.trilinear_backward(q, up)
    bd0, bg0 = b.query(q, mi)
    for threads in (64, 128, 256, 512):
        for cap in (1, 8, 32):
            gvx.set_query_config(threads, cap)
            d, g = m.trilinear(q)
            assert torch.equal(d, d0) and torch.equal(g, g0), (threads, cap)
            assert torch.equal(m.trilinear_backward(q, up), a0), (threads, cap)
            bd, bg = b.query(q, mi)
            assert torch.equal(bd, bd0) and torch.equal(bg, bg0), (threads, cap)
    for bad in ((96, 16), (256, 0), (256, 65)):
        with pytest.raises(gvx.GvxError):
            gvx.set_query_config(*bad)
    cfg = m.autotune_queries(q, force=True)
    assert cfg["threads"] in (64, 128, 256, 512) and cfg["blocks_per_sm"] in (8, 16, 32) and cfg["ms"] > 0
    assert m.autotune_queries(q) == cfg  # cached for the process
    d, g = m.trilinear(q)
    assert torch.equal(d, d0) and torch.equal(g, g0)
    gvx.set_query_config(256, 16)
