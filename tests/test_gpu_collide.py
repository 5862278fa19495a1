"""GPU parity of BitVoxel insertion, map/list collisions and list building
against the oracle, plus the reference's known answers through the C ABI."""
import numpy as np
import pytest
import torch

import gvx
import oracle
import refgeom

pytestmark = pytest.mark.gpu

DIMS = (89, 123, 74)


def _gbvm(dims, pts, meaning=1):
    m = gvx.BitVectorVoxelMap(dims, 1.0)
    m.insertPointCloud(torch.as_tensor(np.asarray(pts, np.float32)), meaning)
    return m


def _obvm(dims, pts, meaning=1):
    m = oracle.bvm_empty(dims)
    oracle.bvm_insert(m, dims, 1.0, pts, meaning)
    return m


def test_known_answers_map_vs_map():
    pts = refgeom.equidistant_points_fast(10_000, DIMS, 1.0)
    assert _gbvm(DIMS, pts).collideWith(_gbvm(DIMS, pts)) == 10_000
    p1 = refgeom.box_of_points((2.1, 2.1, 2.1), (4.1, 4.1, 4.1), 0.5)
    p2 = refgeom.box_of_points((3.1, 3.1, 3.1), (5.1, 5.1, 5.1), 0.5)
    assert _gbvm(DIMS, p1).collideWith(_gbvm(DIMS, p2)) == 8
    assert _gbvm(DIMS, p1).collideWith(_gbvm(DIMS, p2), 0.1, (-1, 0, -1)) == 18
    assert _gbvm(DIMS, p2).collideWith(_gbvm(DIMS, p1), 0.1, (1, 0, 1)) == 18
    black, white = refgeom.nonoverlapping_checkerboard(10_000, DIMS, 1.0)
    assert _gbvm(DIMS, black).collideWith(_gbvm(DIMS, white)) == 0


@pytest.mark.parametrize("dims,seed", [((64, 64, 64), 0), ((37, 21, 90), 1), ((128, 128, 128), 2)])
def test_map_vs_map_counts_and_marks(dims, seed):
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims) // 4)
    pa = (rng.random((n, 3)) * dims).astype(np.float32)
    pb = (rng.random((n, 3)) * dims).astype(np.float32)
    ga, gb = _gbvm(dims, pa, 1), _gbvm(dims, pb, 200)
    oa, ob = _obvm(dims, pa, 1), _obvm(dims, pb, 200)
    assert np.array_equal(ga.voxels().cpu().numpy(), oa)
    for off in [(0, 0, 0), (1, 0, 0), (-3, 2, 1), (0, 0, 5)]:
        lin = off[2] * dims[0] * dims[1] + off[1] * dims[0] + off[0]
        want = oracle.bvm_collide(oa, ob, lin)
        assert ga.collideWith(gb, 1.0, off) == want, off
        assert np.array_equal(ga.voxels().cpu().numpy(), oa), off


def test_free_bit_does_not_collide():
    dims = (16, 16, 16)
    pts = np.array([[1.5, 1.5, 1.5], [3.5, 3.5, 3.5]], np.float32)
    a = _gbvm(dims, pts, 0)   # eBVM_FREE only
    b = _gbvm(dims, pts, 1)
    assert a.collideWith(b) == 0
    a.insertPointCloud(torch.as_tensor(pts[:1]), 255)
    assert a.collideWith(b) == 1


def _glist_from_boxes():
    lst = gvx.BitVectorVoxelList(DIMS, 1.0)
    for (lo, hi), mean in zip([((1.1,) * 3, (3.9,) * 3), ((2.1,) * 3, (4.9,) * 3)], (11, 12)):
        lst.insertPointCloud(torch.as_tensor(refgeom.box_of_points(lo, hi, 0.1)), mean)
    return lst


def test_list_build_matches_oracle():
    lst = _glist_from_boxes()
    ids_o, vox_o = None, None
    for (lo, hi), mean in zip([((1.1,) * 3, (3.9,) * 3), ((2.1,) * 3, (4.9,) * 3)], (11, 12)):
        ids_o, vox_o = oracle.list_insert(ids_o, vox_o, DIMS, 1.0, refgeom.box_of_points(lo, hi, 0.1), mean)
    assert lst.getDimensions() == 46
    assert np.array_equal(lst.ids().cpu().numpy().view(np.uint32), ids_o)
    assert np.array_equal(lst.voxels().cpu().numpy(), vox_o)
    rng = np.random.default_rng(4)
    pts = (rng.random((200_000, 3)) * 120 - 10).astype(np.float32)
    lst.insertPointCloud(torch.as_tensor(pts), 77)
    ids_o, vox_o = oracle.list_insert(ids_o, vox_o, DIMS, 1.0, pts, 77)
    assert np.array_equal(lst.ids().cpu().numpy().view(np.uint32), ids_o)
    assert np.array_equal(lst.voxels().cpu().numpy(), vox_o)


def test_list_known_answers():
    lst = _glist_from_boxes()
    bmap = gvx.BitVectorVoxelMap(DIMS, 1.0)
    for lo, hi in [((1.1,) * 3, (3.9,) * 3), ((2.1,) * 3, (4.9,) * 3)]:
        bmap.insertPointCloud(torch.as_tensor(refgeom.box_of_points(lo, hi, 0.1)), 1)
    assert lst.collideWith(bmap) == 46
    assert (lst.voxels().cpu().numpy().reshape(-1, 32)[:, 0] & 4).all()
    assert lst.collideWith(_glist_from_boxes()) == 46
    box = refgeom.box_of_points((1.1,) * 3, (3.9,) * 3, 0.1)
    one = gvx.BitVectorVoxelList(DIMS, 1.0)
    one.insertPointCloud(torch.as_tensor(box), 1)
    bm = _gbvm(DIMS, box)
    for shift, want in [(0, 27), (1, 18), (2, 9), (3, 0)]:
        assert one.collideWith(bm, 1.0, (shift, 0, 0)) == want
    other_dims = gvx.BitVectorVoxelMap((10, 10, 10), 1.0)
    with pytest.raises(gvx.GvxError):
        one.collideWith(other_dims)
    with pytest.raises(gvx.GvxError):
        one.collideWith(one, 1.0, (1, 0, 0))


def test_list_vs_map_random_with_offsets():
    dims = (64, 64, 64)
    rng = np.random.default_rng(9)
    ids = np.unique(rng.integers(0, 64 ** 3, size=30_000)).astype(np.uint32)
    vox = np.zeros((ids.shape[0], 32), np.uint8)
    vox[:, 0] = rng.choice(np.array([1, 2, 3, 0], np.uint8), size=ids.shape[0])  # some entries only eBVM_FREE
    vox = vox.reshape(-1)
    mp = (rng.random((60_000, 3)) * 64).astype(np.float32)
    om = _obvm(dims, mp, 9)
    gm = _gbvm(dims, mp, 9)
    lst = gvx.BitVectorVoxelList(dims, 1.0)
    for off in [(0, 0, 0), (2, -1, 0), (0, 0, -7)]:
        lst.set(torch.as_tensor(ids.astype(np.int64)), torch.as_tensor(vox).cuda())
        lin = off[2] * 64 * 64 + off[1] * 64 + off[0]
        v = vox.copy()
        want = oracle.list_collide_map(ids, v, om, lin)
        assert lst.collideWith(gm, 1.0, off) == want
        assert np.array_equal(lst.voxels().cpu().numpy(), v)


def test_batched_lists_equal_per_list_counts():
    dims = (64, 64, 64)
    rng = np.random.default_rng(12)
    lengths = np.concatenate([[0, 1, 5], rng.integers(10, 3000, size=60), [0]])
    ids, offs = [], [0]
    for L in lengths:
        v = np.unique(rng.integers(0, 64 ** 3, size=int(L))).astype(np.uint32)
        ids.append(v)
        offs.append(offs[-1] + v.shape[0])
    ids = np.concatenate(ids)
    offs = np.asarray(offs, np.uint64)
    vox = np.zeros((ids.shape[0], 32), np.uint8)
    vox[:, 1] = 1  # meaning 8
    vox = vox.reshape(-1)
    mp = (rng.random((80_000, 3)) * 64).astype(np.float32)
    om = _obvm(dims, mp, 1)
    gm = _gbvm(dims, mp, 1)
    want = oracle.lists_collide_map_omp(ids, vox, offs, om)
    for k in range(len(lengths)):
        a, b = int(offs[k]), int(offs[k + 1])
        assert want[k] == oracle.list_collide_map(ids[a:b], vox[a * 32:b * 32].copy(), om)
    got = gvx.lists_collide_map(torch.as_tensor(ids.astype(np.int64)).to(torch.int32).cuda(),
                                torch.as_tensor(vox).cuda(), torch.as_tensor(offs.astype(np.int64)).cuda(), gm)
    assert np.array_equal(got.cpu().numpy().astype(np.uint64), want)


@pytest.mark.parametrize("dims,shifted", [((64, 64, 64), False), ((24, 20, 17), False), ((24, 20, 17), True)])
def test_batched_lists_both_paths_with_marks(dims, shifted):
    """The batched call gathers a map voxel per entry (64^3: fewer entries than
    half the voxels) or first reduces the map to occupancy bits (24x20x17:
    many entries per voxel; its ids are read 16 bytes at a time when aligned,
    4 at a time when the id array starts 4 bytes off -- `shifted`); every path
    gives the oracle's counts and marks, with empty lists, free-only entries
    and ids beyond the map."""
    nvox = int(np.prod(dims))
    rng = np.random.default_rng(21)
    lengths = np.concatenate([[0, 3], rng.integers(10, 2500, size=40), [0, 1]])
    ids, offs = [], [0]
    for L in lengths:
        v = np.unique(rng.integers(0, nvox + 50, size=int(L))).astype(np.uint32)
        ids.append(v)
        offs.append(offs[-1] + v.shape[0])
    ids = np.concatenate(ids)
    offs = np.asarray(offs, np.uint64)
    vox = np.zeros((ids.shape[0], 32), np.uint8)
    vox[:, 1] = 1  # meaning 8
    free = rng.random(ids.shape[0]) < 0.1
    vox[free] = 0
    vox[free, 0] = 1  # eBVM_FREE only: never collides
    vox = vox.reshape(-1)
    mp = (rng.random((nvox // 3, 3)) * dims).astype(np.float32)
    # the map: occupied points, then free-only points
    gmap = _gbvm(dims, mp, 1)
    free_pts = (np.random.default_rng(99).random((nvox // 10, 3)) * dims).astype(np.float32)
    om = _obvm(dims, mp, 1)
    oracle.bvm_insert(om, dims, 1.0, free_pts, 0)
    gmap.insertPointCloud(torch.as_tensor(free_pts), 0)
    assert np.array_equal(gmap.voxels().cpu().numpy(), om)
    want_vox = vox.copy()
    want = []
    for k in range(len(lengths)):
        a, b = int(offs[k]), int(offs[k + 1])
        seg = want_vox[a * 32:b * 32].copy()
        want.append(oracle.list_collide_map(ids[a:b], seg, om, 0, True))
        want_vox[a * 32:b * 32] = seg
    assert (2 * ids.shape[0] >= nvox) == (dims != (64, 64, 64))
    dv = torch.as_tensor(vox).cuda()
    dids = torch.as_tensor(np.concatenate([[0], ids]).astype(np.int64)).to(torch.int32).cuda()
    dids = dids[1:] if shifted else dids[1:].clone()
    assert (dids.data_ptr() % 16 == 4) == shifted
    got = gvx.lists_collide_map(dids, dv, torch.as_tensor(offs.astype(np.int64)).cuda(), gmap, mark=True)
    assert got.cpu().numpy().tolist() == want and sum(want) > 0
    assert np.array_equal(dv.cpu().numpy(), want_vox)
