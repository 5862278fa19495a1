"""Parity at the benchmark configurations' full sizes: every count and map the
bench sections report is compared with the oracle (OpenMP C restatement) or
with gpu-voxels' own kernels on the same inputs.

  C2  512^3 depth-scene BitVectorVoxelMap collideWith the 512^3 capsule map:
      count and eBVM_COLLISION marks (the 64-bit voxel offsets of a 4 GiB map);
      at 512 x 512 x 511 (the largest map the reference's 32-bit byte count
      allows) also against the reference's own collide kernel.
  C3  all 4096 swept-volume lists of 2k..200k ids against the 256^3 scene:
      per-list counts against the oracle and against the reference's list
      kernel run once per list, and the marks the reference leaves.
  C5  the 64 uneven maps (dims log-uniform in [64, 384]) through the batched
      voxelise + EDT, the CUDA-graph replay and the batched insert + EDT:
      every map bit for bit against the oracle's EDT.
"""
import numpy as np
import pytest
import torch

import gvx
import oracle
import workloads
from gvx.batch import Batch
from gpu_helpers import first_mismatch, to_u32

pytestmark = pytest.mark.gpu

C2_DIMS, C2_SIDE = (512, 512, 512), 0.005


@pytest.fixture(scope="module")
def c2_inputs():
    return workloads.c2_points(), workloads.capsule_points()


def _gvx_bvm(dims, side, pts, meaning):
    m = gvx.BitVectorVoxelMap(dims, side)
    m.insertPointCloud(torch.as_tensor(pts).cuda(), meaning)
    return m


def _oracle_bvm(dims, side, pts, meaning):
    m = oracle.bvm_empty(dims)
    oracle.bvm_insert(m, dims, side, pts, meaning)
    return m


def test_c2_collide_512cubed_count_and_marks(c2_inputs):
    pts, caps = c2_inputs
    scene = _gvx_bvm(C2_DIMS, C2_SIDE, pts, 1)
    capsules = _gvx_bvm(C2_DIMS, C2_SIDE, caps, 4)
    o_scene = _oracle_bvm(C2_DIMS, C2_SIDE, pts, 1)
    o_caps = _oracle_bvm(C2_DIMS, C2_SIDE, caps, 4)
    assert np.array_equal(capsules.voxels().cpu().numpy(), o_caps)
    count = scene.collideWith(capsules)
    want = oracle.bvm_collide(o_scene, o_caps)  # marks o_scene
    assert count == want and want > 0
    assert np.array_equal(scene.voxels().cpu().numpy(), o_scene), "eBVM_COLLISION marks differ"


def test_c2_collide_512x512x511_against_reference_kernel(c2_inputs):
    R = oracle.ref_lib()
    if R is None:
        pytest.skip("oracle/_ref/libgvref.so not built (needs the reference source tree at build time)")
    import ctypes

    dims = (512, 512, 511)
    pts, caps = c2_inputs
    o_scene = _oracle_bvm(dims, C2_SIDE, pts, 1)
    o_caps = _oracle_bvm(dims, C2_SIDE, caps, 4)
    r_scene = o_scene.copy()
    cnt = ctypes.c_uint64(0)
    assert R.ref_bvm_collide(r_scene, o_caps, int(np.prod(dims)), ctypes.byref(cnt)) == 0
    want = oracle.bvm_collide(o_scene, o_caps)
    assert cnt.value == want and want > 0
    assert np.array_equal(r_scene, o_scene)
    scene = _gvx_bvm(dims, C2_SIDE, pts, 1)
    capsules = _gvx_bvm(dims, C2_SIDE, caps, 4)
    assert scene.collideWith(capsules) == want
    assert np.array_equal(scene.voxels().cpu().numpy(), r_scene)


def _c3_lists():
    """The bench's C3 lists: 4096 lists of 2k..200k ids (sorted, unique) on
    the 256^3 scene's map, list k's voxels carrying meaning 4 + k % 200."""
    sc = workloads.c3_scene()
    nvox = int(np.prod(sc.dims))
    ids, offs = workloads.c3_lists_device(workloads.list_lengths(), nvox)
    owner = torch.repeat_interleave(torch.arange(offs.shape[0] - 1, device="cuda"), offs[1:] - offs[:-1])
    meaning = 4 + owner % 200
    vox = torch.zeros(ids.numel(), 32, dtype=torch.uint8, device="cuda")
    vox.scatter_(1, (meaning // 8).unsqueeze(1), (1 << (meaning % 8)).to(torch.uint8).unsqueeze(1))
    bmap = _gvx_bvm(sc.dims, sc.side, sc.points, 1)
    return sc, ids, vox.reshape(-1), offs, bmap


def test_c3_all_4096_lists_counts_against_oracle_and_reference():
    sc, ids, vox, offs, bmap = _c3_lists()
    assert offs.shape[0] == 4097 and ids.numel() > 100_000_000
    counts = gvx.lists_collide_map(ids, vox, offs, bmap)  # the bench's call (no marks)
    ids_h = ids.cpu().numpy().view(np.uint32)
    vox_h = vox.cpu().numpy()
    offs_h = offs.cpu().numpy().astype(np.uint64)
    map_h = bmap.voxels().cpu().numpy()
    assert np.array_equal(map_h, _oracle_bvm(sc.dims, sc.side, sc.points, 1))
    want = oracle.lists_collide_map_omp(ids_h, vox_h, offs_h, map_h)
    got = counts.cpu().numpy().astype(np.uint64)
    assert np.array_equal(got, want), f"{int((got != want).sum())} lists differ"
    assert int(want.sum()) > 0
    R = oracle.ref_lib()
    if R is None:
        return
    ref_counts = np.zeros(4096, dtype=np.uint64)
    ref_vox = vox_h.copy()
    assert R.ref_lists_collide_map(ids_h, ref_vox, offs_h, 4096, map_h, np.asarray(sc.dims, np.uint32),
                                   np.zeros(3, np.int32), ref_counts) == 0
    assert np.array_equal(ref_counts, want)
    gvx.lists_collide_map(ids, vox, offs, bmap, mark=True, counts=counts)
    assert np.array_equal(counts.cpu().numpy().astype(np.uint64), want)
    assert np.array_equal(vox.cpu().numpy(), ref_vox), "eBVM_COLLISION marks differ from the reference kernel's"


def test_list_collide_with_offsets_against_reference_kernel():
    """Random lists (ids beyond the map, free-only entries) through the single-
    list collideWith at four offsets: counts and marks equal the reference
    kernel's, launched once per list as BitVoxelList::collideWith does."""
    from golden_cases import LIST_CASE, linear_offset, list_inputs

    R = oracle.ref_lib()
    bmap, ids, vox, offs = list_inputs(LIST_CASE)
    dims = LIST_CASE["dims"]
    g_map = gvx.BitVectorVoxelMap(dims, 1.0)
    import ctypes
    ptr = ctypes.c_void_p()
    gvx._abi.call("gvx_bvm_info", g_map.handle, None, None, ctypes.byref(ptr))
    dev = gvx.maps._device_view_u8(ptr.value, bmap.shape[0])
    dev.copy_(torch.as_tensor(bmap))
    assert np.array_equal(g_map.voxels().cpu().numpy(), bmap)
    for off in LIST_CASE["offsets"]:
        lin = linear_offset(dims, off)
        ref_counts = np.zeros(offs.shape[0] - 1, dtype=np.uint64)
        ref_vox = vox.copy()
        if R is not None:
            assert R.ref_lists_collide_map(ids, ref_vox, offs, ref_counts.shape[0], bmap, np.asarray(dims, np.uint32),
                                           np.asarray(off, np.int32), ref_counts) == 0
        for l in range(offs.shape[0] - 1):
            a, b = int(offs[l]), int(offs[l + 1])
            seg = vox[a * 32:b * 32].copy()
            want = oracle.list_collide_map(ids[a:b], seg, bmap, lin, True)
            lst = gvx.BitVectorVoxelList(dims, 1.0)
            lst.set(torch.as_tensor(ids[a:b].astype(np.int64)).cuda(), torch.as_tensor(vox[a * 32:b * 32]).cuda())
            assert lst.collideWith(g_map, 1.0, off) == want, (off, l)
            assert np.array_equal(lst.voxels().cpu().numpy(), seg), (off, l)
            if R is not None:
                assert int(ref_counts[l]) == want, (off, l)
                assert np.array_equal(ref_vox[a * 32:b * 32], seg), (off, l)


@pytest.fixture(scope="module")
def c5():
    scenes = workloads.c5_maps()
    want = []
    for s in scenes:
        m = oracle.dvm_empty(s.dims)
        oracle.dvm_insert(m, s.dims, s.side, s.points)
        oracle.pba(m, s.dims)
        want.append(m)
    pts = torch.as_tensor(np.concatenate([s.points for s in scenes]).astype(np.float32)).cuda()
    offs = np.zeros(len(scenes) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([s.points.shape[0] for s in scenes])
    return scenes, want, pts, torch.as_tensor(offs).cuda()


def _check_maps(maps, want, scenes, what):
    for k, (m, w, s) in enumerate(zip(maps, want, scenes)):
        got = to_u32(m.data())
        assert np.array_equal(got, w), (what, k, s.dims, first_mismatch(got, w, s.dims))


def test_c5_64_uneven_maps_batched_voxelize_edt_and_graph_replay(c5):
    scenes, want, pts, offs = c5
    assert len(scenes) == 64
    maps = [gvx.DistanceVoxelMap(s.dims, s.side) for s in scenes]
    b = Batch(maps)
    b.voxelize_edt(pts, offs)
    assert b.edt_check() == 0
    _check_maps(maps, want, scenes, "voxelize_edt")
    for m in maps:
        m.clearMap()
    q = torch.full((64, 3), 0.02, dtype=torch.float32, device="cuda")
    qm = torch.arange(64, dtype=torch.int32, device="cuda")
    b.capture(pts, offs, q, qm)
    b.replay()
    b.replay()
    assert b.edt_check() == 0
    _check_maps(maps, want, scenes, "graph replay")


def test_c5_64_uneven_maps_batched_insert_then_edt(c5):
    scenes, want, pts, offs = c5
    maps = [gvx.DistanceVoxelMap(s.dims, s.side) for s in scenes]
    b = Batch(maps)
    b.clear()
    b.insert(pts, offs)
    b.edt()
    assert b.edt_check() == 0
    _check_maps(maps, want, scenes, "insert + edt")
