"""insertMetaPointCloudWithSelfCollisionCheck in the oracle, pinned by the
known answers of the reference's own test (GV/test/testing_voxelmap.cu,
selfcollision_metapointcloud: default fixture dims 89 x 123 x 74, side 1)."""
import numpy as np
import pytest

import oracle
import refgeom

DIMS = (89, 123, 74)


def _boxes(corners, j):
    return [refgeom.box_of_points(lo, hi, 1.0 / j) for lo, hi in corners]


COLLIDING = [((2.1,) * 3, (5.1,) * 3), ((4.1,) * 3, (7.1,) * 3), ((6.1,) * 3, (9.1,) * 3), ((10.1,) * 3, (12.1,) * 3)]
NONCOLLIDING = [((30.1,) * 3, (32.1,) * 3), ((40.1,) * 3, (43.1,) * 3), ((60.1,) * 3, (64.1,) * 3),
                ((65.1,) * 3, (68.1,) * 3)]


def _all_but(*bits):
    m = np.full(32, 0xFF, dtype=np.uint8)
    for b in bits:
        m[b >> 3] &= ~np.uint8(1 << (b & 7))
    return m


@pytest.mark.parametrize("j", [2, 10])  # the reference runs j = 2 and j = 10 (1/j point spacing)
def test_reference_known_answers(j):
    m = oracle.bvm_empty(DIMS)
    # part 1: default meanings and masks
    hit, _, out = oracle.bvm_insert_meta_self_coll(m, DIMS, 1.0, _boxes(COLLIDING, j))
    assert hit is True and not out
    hit, _, _ = oracle.bvm_insert_meta_self_coll(m, DIMS, 1.0, _boxes(NONCOLLIDING, j))
    assert hit is False
    m[:] = 0
    # part 2: meanings 51..54; cloud 0 ignores cloud 1 and cloud 1 ignores cloud 0
    meanings = [51, 52, 53, 54]
    masks = np.stack([_all_but(2, 52, 51), _all_but(2, 51, 52), _all_but(2, 53), _all_but(2, 54)])
    hit, coll, _ = oracle.bvm_insert_meta_self_coll(m, DIMS, 1.0, _boxes(COLLIDING, j), meanings, masks)
    bits = {b for b in range(256) if coll[b >> 3] >> (b & 7) & 1}
    assert hit is True and bits == {52, 53}
    masks = np.stack([_all_but(2, 51), _all_but(2, 52), _all_but(2, 53), _all_but(2, 54)])
    hit, coll, _ = oracle.bvm_insert_meta_self_coll(m, DIMS, 1.0, _boxes(NONCOLLIDING, j), meanings, masks)
    assert hit is False and not coll.any()


def test_marks_and_outside_flag():
    dims = (8, 8, 8)
    m = oracle.bvm_empty(dims)
    a = np.array([[1.5, 1.5, 1.5], [2.5, 2.5, 2.5]], np.float32)
    b = np.array([[2.5, 2.5, 2.5], [20.0, 1.0, 1.0]], np.float32)  # second point outside
    hit, coll, out = oracle.bvm_insert_meta_self_coll(m, dims, 1.0, [a, b])
    assert hit and out
    bits = {k for k in range(256) if coll[k >> 3] >> (k & 7) & 1}
    assert bits == {4, 5}  # cloud 1 met cloud 0's meaning in voxel (2,2,2) and reports its own
    v = m.reshape(-1, 32)[2 * 64 + 2 * 8 + 2]
    assert v[0] & (1 << 2) and v[0] & (1 << 4) and v[0] & (1 << 5)  # eBVM_COLLISION + both meanings
    assert not (m.reshape(-1, 32)[1 * 64 + 1 * 8 + 1][0] & (1 << 2))  # cloud 0 alone: no collision mark
