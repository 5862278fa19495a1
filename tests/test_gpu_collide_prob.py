"""collideWith against a ProbVoxelMap (DefaultCollider: occupancy >=
floatToProbability(threshold), BitVoxel holding a meaning other than
eBVM_FREE), for a BitVectorVoxelMap and a BitVectorVoxelList: counts and
eBVM_COLLISION marks against the oracle at several thresholds (clamped ones
included) and offsets, and against gpu-voxels' own kernels where built."""
import ctypes

import numpy as np
import pytest
import torch

import gvx
import oracle
from golden_cases import linear_offset

pytestmark = pytest.mark.gpu

DIMS = (64, 48, 40)
THRESHOLDS = [-0.5, 0.0, 0.3, 0.55, 0.9, 1.0, 1.7]
OFFSETS = [(0, 0, 0), (1, 0, 0), (-3, 2, 1), (0, 0, 5)]


def _prob_scene(seed=31):
    """A ProbVoxelMap with varied occupancies: points inserted as occupied or
    free, some voxels many times; same inserts on the GPU and in the oracle."""
    rng = np.random.default_rng(seed)
    pm = gvx.ProbVoxelMap(DIMS, 1.0)
    om = oracle.pvm_empty(DIMS)
    for rep in range(6):
        for meaning in (gvx.eBVM_OCCUPIED, gvx.eBVM_FREE):
            pts = (rng.random((4000, 3)) * [DIMS[0], DIMS[1], DIMS[2] / 3 * (1 + rep % 3)]).astype(np.float32)
            pm.insertPointCloud(torch.as_tensor(pts), meaning)
            oracle.pvm_insert(om, DIMS, 1.0, pts, meaning)
    got = pm.data().cpu().numpy().view(np.int8)
    assert np.array_equal(got, om)
    assert len(np.unique(om)) > 5
    return pm, om


def _bit_scene(seed=32):
    rng = np.random.default_rng(seed)
    pts = (rng.random((30000, 3)) * DIMS).astype(np.float32)
    free = (rng.random((6000, 3)) * DIMS).astype(np.float32)
    g = gvx.BitVectorVoxelMap(DIMS, 1.0)
    g.insertPointCloud(torch.as_tensor(pts), 9)
    g.insertPointCloud(torch.as_tensor(free), gvx.eBVM_FREE)
    o = oracle.bvm_empty(DIMS)
    oracle.bvm_insert(o, DIMS, 1.0, pts, 9)
    oracle.bvm_insert(o, DIMS, 1.0, free, gvx.eBVM_FREE)
    assert np.array_equal(g.voxels().cpu().numpy(), o)
    return g, o


def test_bitvoxelmap_collide_with_prob_map():
    pm, om = _prob_scene()
    for thr in THRESHOLDS:
        for off in OFFSETS:
            g, o = _bit_scene()
            want = oracle.bvm_collide_pvm(o, om, thr, linear_offset(DIMS, off))
            assert g.collideWith(pm, thr, off) == want, (thr, off)
            assert np.array_equal(g.voxels().cpu().numpy(), o), (thr, off)
    # a ProbVoxelMap of other dims is refused
    other = gvx.ProbVoxelMap((8, 8, 8), 1.0)
    with pytest.raises(gvx.GvxError):
        g.collideWith(other)


def test_bitvoxellist_collide_with_prob_map():
    from golden_cases import LIST_CASE, list_inputs

    pm, om = _prob_scene()
    _, ids, vox, offs = list_inputs(LIST_CASE)
    for thr in (0.0, 0.55, 1.0):
        for off in OFFSETS:
            lin = linear_offset(DIMS, off)
            for l in range(offs.shape[0] - 1):
                a, b = int(offs[l]), int(offs[l + 1])
                seg = vox[a * 32:b * 32].copy()
                want = oracle.list_collide_pvm(ids[a:b], seg, om, thr, lin)
                lst = gvx.BitVectorVoxelList(DIMS, 1.0)
                lst.set(torch.as_tensor(ids[a:b].astype(np.int64)).cuda(), torch.as_tensor(vox[a * 32:b * 32]).cuda())
                assert lst.collideWith(pm, thr, off) == want, (thr, off, l)
                assert np.array_equal(lst.voxels().cpu().numpy(), seg), (thr, off, l)


def test_prob_map_collisions_against_reference_kernels():
    R = oracle.ref_lib()
    if R is None:
        pytest.skip("oracle/_ref/libgvref.so not built (needs the reference source tree at build time)")
    from golden_cases import LIST_CASE, list_inputs

    _, om = _prob_scene()
    _, o = _bit_scene()
    _, ids, vox, offs = list_inputs(LIST_CASE)
    for thr in THRESHOLDS:
        r_self = o.copy()
        cnt = ctypes.c_uint64(0)
        assert R.ref_bvm_collide_pvm(r_self, om, int(np.prod(DIMS)), float(thr), ctypes.byref(cnt)) == 0
        o_self = o.copy()
        assert oracle.bvm_collide_pvm(o_self, om, thr) == cnt.value, thr
        assert np.array_equal(o_self, r_self), thr
        for off in OFFSETS:
            for l in range(offs.shape[0] - 1):
                a, b = int(offs[l]), int(offs[l + 1])
                r_seg = vox[a * 32:b * 32].copy()
                c = ctypes.c_uint64(0)
                assert R.ref_list_collide_pvm(ids[a:b], r_seg, b - a, om, np.asarray(DIMS, np.uint32),
                                              np.asarray(off, np.int32), float(thr), ctypes.byref(c)) == 0
                o_seg = vox[a * 32:b * 32].copy()
                assert oracle.list_collide_pvm(ids[a:b], o_seg, om, thr, linear_offset(DIMS, off)) == c.value
                assert np.array_equal(o_seg, r_seg)
