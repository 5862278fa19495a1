"""Typed collisions on the GPU against the oracle: the colliding types, the
counts and the eBVM_COLLISION marks, for map vs map, map vs ProbVoxelMap,
list vs map / ProbVoxelMap / list and the type-mask form."""
import numpy as np
import pytest
import torch

import gvx
import oracle

pytestmark = pytest.mark.gpu

DIMS = (48, 40, 36)


def _random_bits(rng, n, density=0.02):
    """n 32-byte voxels with a few random meaning bits each (some empty)."""
    v = np.zeros((n, 32), np.uint8)
    bits = rng.random((n, 256)) < density
    for k in range(256):
        v[:, k >> 3] |= (bits[:, k].astype(np.uint8) << (k & 7))
    v[rng.random(n) < 0.3] = 0
    return v.reshape(-1)


def _bvm_from(vox):
    m = gvx.BitVectorVoxelMap(DIMS, 1.0)
    m.voxels().copy_(torch.as_tensor(vox).cuda())
    return m


def test_map_vs_map_types():
    rng = np.random.default_rng(0)
    n = int(np.prod(DIMS))
    a, b = _random_bits(rng, n), _random_bits(rng, n)
    ga, gb = _bvm_from(a), _bvm_from(b)
    count, types = ga.collideWithTypes(gb)
    want_n, want_t = oracle.bvm_collide_types(a, b)
    assert count == want_n and np.array_equal(types, want_t)
    assert np.array_equal(ga.voxels().cpu().numpy(), a)  # marks


def test_map_vs_prob_types():
    rng = np.random.default_rng(1)
    n = int(np.prod(DIMS))
    a = _random_bits(rng, n)
    p = gvx.ProbVoxelMap(DIMS, 1.0)
    occ = rng.integers(-128, 128, n).astype(np.int8)
    p.data().copy_(torch.as_tensor(occ).cuda())
    for thr in (0.5, 0.9, 1.0, 0.0):
        ga = _bvm_from(a)
        ref = a.copy()
        count, types = ga.collideWithTypes(p, thr)
        want_n, want_t = oracle.bvm_collide_types_pvm(ref, occ, thr)
        assert count == want_n and np.array_equal(types, want_t), thr
        assert np.array_equal(ga.voxels().cpu().numpy(), ref)


def _list(rng, k):
    n = int(np.prod(DIMS))
    ids = np.unique(rng.integers(0, n, k)).astype(np.uint32)
    vox = _random_bits(rng, ids.size, 0.05)
    lst = gvx.BitVectorVoxelList(DIMS, 1.0)
    lst.set(torch.as_tensor(ids.astype(np.int32)).cuda(), torch.as_tensor(vox).cuda())
    return lst, ids, vox


@pytest.mark.parametrize("offset", [(0, 0, 0), (3, -2, 1)])
def test_list_vs_map_prob_and_mask(offset):
    rng = np.random.default_rng(2)
    n = int(np.prod(DIMS))
    lin = offset[0] + offset[1] * DIMS[0] + offset[2] * DIMS[0] * DIMS[1]
    mvox = _random_bits(rng, n, 0.01)
    gmap = _bvm_from(mvox)
    lst, ids, vox = _list(rng, 5000)
    count, types = lst.collideWithTypes(gmap, 1.0, offset)
    ref = vox.copy()
    want_n, want_t = oracle.list_collide_types_map(ids, ref, mvox, lin)
    assert count == want_n and np.array_equal(types, want_t)
    assert np.array_equal(lst.voxels().cpu().numpy().reshape(-1), ref)

    occ = rng.integers(-128, 128, n).astype(np.int8)
    p = gvx.ProbVoxelMap(DIMS, 1.0)
    p.data().copy_(torch.as_tensor(occ).cuda())
    lst2, ids2, vox2 = _list(rng, 4000)
    count, types = lst2.collideWithTypes(p, 12.5, offset)
    ref2 = vox2.copy()
    want_n, want_t = oracle.list_collide_types_map(ids2, ref2, occ, lin, prob_threshold=12.5)
    assert count == want_n and np.array_equal(types, want_t)
    assert np.array_equal(lst2.voxels().cpu().numpy().reshape(-1), ref2)

    lst3, ids3, vox3 = _list(rng, 4000)
    mask = np.zeros(32, np.uint8)
    mask[2] = 0xF0
    mask[17] = 0x0F
    count = lst3.collideWithTypeMask(gmap, mask, 1.0, offset)
    ref3 = vox3.copy()
    want_n, _ = oracle.list_collide_types_map(ids3, ref3, mvox, lin, mask=mask)
    assert count == want_n
    assert np.array_equal(lst3.voxels().cpu().numpy().reshape(-1), ref3)


def test_list_vs_list_types():
    rng = np.random.default_rng(3)
    a, ida, va = _list(rng, 6000)
    b, idb, vb = _list(rng, 3000)
    count, types = a.collideWithTypes(b)
    want_n, want_t = oracle.list_collide_types_list(ida, va, idb, vb)
    assert count == want_n and np.array_equal(types, want_t)
