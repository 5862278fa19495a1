"""insertMetaPointCloudWithSelfCollisionCheck on the GPU against the oracle:
the reference test's known answers, random multi-link clouds over existing
map content, and user meanings and masks (masks clear the sub-cloud's own
meaning and eBVM_COLLISION, as the reference's defaults do: with those bits
kept the reference's own result depends on its threads' timing)."""
import numpy as np
import pytest
import torch

import gvx
import oracle
from test_oracle_meta import COLLIDING, DIMS, NONCOLLIDING, _all_but, _boxes

pytestmark = pytest.mark.gpu


def _bits(c):
    return {b for b in range(256) if c[b >> 3] >> (b & 7) & 1}


@pytest.mark.parametrize("j", [2, 10])
def test_reference_known_answers(j):
    m = gvx.BitVectorVoxelMap(DIMS, 1.0)
    hit, _ = m.insertMetaPointCloudWithSelfCollisionCheck(_boxes(COLLIDING, j))
    assert hit is True
    hit, _ = m.insertMetaPointCloudWithSelfCollisionCheck(_boxes(NONCOLLIDING, j))
    assert hit is False
    m.clearMap()
    meanings = [51, 52, 53, 54]
    masks = np.stack([_all_but(2, 52, 51), _all_but(2, 51, 52), _all_but(2, 53), _all_but(2, 54)])
    hit, coll = m.insertMetaPointCloudWithSelfCollisionCheck(_boxes(COLLIDING, j), meanings, masks)
    assert hit is True and _bits(coll) == {52, 53}
    masks = np.stack([_all_but(2, 51), _all_but(2, 52), _all_but(2, 53), _all_but(2, 54)])
    hit, coll = m.insertMetaPointCloudWithSelfCollisionCheck(_boxes(NONCOLLIDING, j), meanings, masks)
    assert hit is False and not coll.any()


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_links_match_oracle(seed):
    rng = np.random.default_rng(seed)
    dims = (64, 80, 50)
    env = (rng.random((3000, 3)) * np.asarray(dims) * 0.05).astype(np.float32)
    links = []
    for k in range(9):  # overlapping blobs along a chain, a few points outside the map
        c = rng.random(3) * np.asarray(dims) * 0.05
        pts = c + rng.normal(scale=0.2, size=(int(rng.integers(50, 4000)), 3))
        links.append(pts.astype(np.float32))
    links[3][:5] = 1000.0  # beyond the map (negative coordinates land in voxel 0)
    meanings = None if seed == 0 else rng.choice(np.arange(4, 255), size=len(links), replace=False)
    masks = None
    if seed == 2:  # random masks, own meaning and eBVM_COLLISION cleared
        masks = rng.integers(0, 256, size=(len(links), 32)).astype(np.uint8)
        for k, mk in enumerate(meanings):
            masks[k] &= _all_but(2, int(mk))
    want = oracle.bvm_empty(dims)
    oracle.bvm_insert(want, dims, 0.05, env, 1)
    hit_o, coll_o, out_o = oracle.bvm_insert_meta_self_coll(want, dims, 0.05, links, meanings, masks)
    m = gvx.BitVectorVoxelMap(dims, 0.05)
    m.insertPointCloud(torch.as_tensor(env).cuda(), meaning=1)
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    hit, coll = m.insertMetaPointCloudWithSelfCollisionCheck(links, meanings, masks, outside=flag)
    assert hit == hit_o and np.array_equal(coll, coll_o)
    assert bool(flag.item()) == out_o
    assert np.array_equal(m.voxels().cpu().numpy().reshape(-1), want)


@pytest.mark.parametrize("shift", [0, 3, 13, 31, 32, 33, 56])
def test_shift_and_clear_match_oracle(shift):
    """shiftLeftSweptVolumeIDs and clearBits on every voxel of a random map."""
    dims = (33, 17, 9)
    rng = np.random.default_rng(shift)
    raw = rng.integers(0, 256, size=int(np.prod(dims)) * 32).astype(np.uint8)
    m = gvx.BitVectorVoxelMap(dims, 1.0)
    m.voxels().copy_(torch.as_tensor(raw).cuda())
    m.shiftLeftSweptVolumeIDs(shift)
    want = oracle.bvm_shift(raw.copy(), shift)
    assert np.array_equal(m.voxels().cpu().numpy(), want)
    bits = rng.integers(0, 256, size=32).astype(np.uint8)
    m.clearBits(bits)
    oracle.bvm_clear_bits(want, bits)
    assert np.array_equal(m.voxels().cpu().numpy(), want)
    m.clearBitVoxelMeaning(200)
    oracle.bvm_clear_bits(want, _all_but(*[b for b in range(256) if b != 200]))
    assert np.array_equal(m.voxels().cpu().numpy(), want)


def test_shift_above_56_is_refused():
    m = gvx.BitVectorVoxelMap((4, 4, 4), 1.0)
    m.insertPointCloud(torch.tensor([[1.5, 1.5, 1.5]], device="cuda"), meaning=100)
    before = m.voxels().clone()
    with pytest.raises(Exception):
        m.shiftLeftSweptVolumeIDs(57)
    assert torch.equal(m.voxels(), before)


def test_list_shift_and_clear_match_oracle():
    dims = (40, 30, 20)
    rng = np.random.default_rng(3)
    lst = gvx.BitVectorVoxelList(dims, 1.0)
    for meaning in (7, 40, 200, 250):
        lst.insertPointCloud(torch.as_tensor((rng.random((500, 3)) * np.asarray(dims)).astype(np.float32)).cuda(),
                             meaning=meaning)
    vox = lst.voxels().cpu().numpy().reshape(-1).copy()
    lst.shiftLeftSweptVolumeIDs(13)
    oracle.bvm_shift(vox, 13)
    assert np.array_equal(lst.voxels().cpu().numpy().reshape(-1), vox)
    lst.clearBitVoxelMeaning(237)  # 250 - 13
    b = np.zeros(32, np.uint8)
    b[237 >> 3] = 1 << (237 & 7)
    oracle.bvm_clear_bits(vox, b)
    assert np.array_equal(lst.voxels().cpu().numpy().reshape(-1), vox)


def test_clone_every_map_type_and_refusals():
    """TemplateVoxelMap::clone (GV/voxelmap/TemplateVoxelMap.hpp:1101-1120)."""
    dims = (31, 27, 19)
    rng = np.random.default_rng(11)
    pts = torch.as_tensor((rng.random((3000, 3)) * np.asarray(dims) * 0.05).astype(np.float32)).cuda()
    a, b = gvx.DistanceVoxelMap(dims, 0.05), gvx.DistanceVoxelMap(dims, 0.05)
    a.voxelize_edt(pts)
    b.clone(a)
    assert torch.equal(a.data(), b.data())
    with pytest.raises(ValueError):
        gvx.DistanceVoxelMap((31, 27, 18), 0.05).clone(a)
    with pytest.raises(ValueError):
        gvx.DistanceVoxelMap(dims, 0.04).clone(a)
    ba, bb = gvx.BitVectorVoxelMap(dims, 0.05), gvx.BitVectorVoxelMap(dims, 0.05)
    ba.insertPointCloud(pts, 9)
    bb.clone(ba)
    assert torch.equal(ba.voxels(), bb.voxels())
    pa, pb = gvx.ProbVoxelMap(dims, 0.05), gvx.ProbVoxelMap(dims, 0.05)
    pa.insertPointCloud(pts)
    pb.clone(pa)
    assert torch.equal(pa.data(), pb.data())
