"""CPU tests of the oracle: the reference's own known answers, an independent
exact EDT, the literal launch order vs the generalised sweeps, and the
voxelisation edge cases.  No GPU needed."""
import math

import numpy as np
import pytest
from scipy import ndimage

import oracle
import refgeom

DV_UNINIT = oracle.DV_UNINIT


def _inserted(dims, pts, side=1.0):
    m = oracle.dvm_empty(dims)
    oracle.dvm_insert(m, dims, side, pts)
    return m


def _exact_sqdist(inserted, dims):
    """Exact squared EDT from scipy (independent of the PBA restatement)."""
    X, Y, Z = dims
    occ = (inserted != DV_UNINIT).reshape(Z, Y, X)
    if not occ.any():
        return np.full(inserted.shape, oracle.INT_MAX, dtype=np.int64)
    d = ndimage.distance_transform_edt(~occ, return_distances=True)
    return np.rint(d.astype(np.float64) ** 2).astype(np.int64).reshape(-1)


def _sites_sqdist(vmap, dims):
    return oracle.sqdist_map(vmap, dims).astype(np.int64)


# ---- voxelisation ---------------------------------------------------------

def test_coord_to_voxel_saturates_like_the_device():
    # mapToVoxels: floor(c / s) then a saturating float->u32 convert
    assert oracle.coord_to_voxel(0.0, 1.0) == 0
    assert oracle.coord_to_voxel(2.999, 1.0) == 2
    assert oracle.coord_to_voxel(3.0, 1.0) == 3
    assert oracle.coord_to_voxel(-0.5, 1.0) == 0       # negative -> voxel 0 (inserted!)
    assert oracle.coord_to_voxel(-1e9, 1.0) == 0
    assert oracle.coord_to_voxel(float("nan"), 1.0) == 0
    assert oracle.coord_to_voxel(1e30, 1.0) == 0xFFFFFFFF
    assert oracle.coord_to_voxel(0.3, 0.1) == int(np.floor(np.float32(0.3) / np.float32(0.1)))


def test_insert_writes_own_coordinates_and_flags_outside():
    dims = (8, 9, 10)
    pts = np.array([[0.5, 0.5, 0.5], [7.9, 8.9, 9.9], [8.0, 0, 0], [-3.0, 2.5, 1.5]], dtype=np.float32)
    m = oracle.dvm_empty(dims)
    outside = oracle.dvm_insert(m, dims, 1.0, pts)
    assert outside
    occ = np.nonzero(m != DV_UNINIT)[0]
    # (0,0,0) from the first point, (7,8,9) from the second, (0,2,1) from the negative x point
    ids = sorted([0, 9 * 10 * 8 - 1, (1 * 9 + 2) * 8 + 0])
    assert occ.tolist() == ids
    x, y, z = oracle.decode_sites(m[occ])
    assert (x == occ % 8).all() and (y == (occ // 8) % 9).all() and (z == occ // 72).all()


# ---- known answers of GV/test/testing_distance.cu -----------------------

def test_distance_extraction_64():
    """distance_extraction (GV/test/testing_distance.cu:129-220)."""
    dims = (64, 64, 64)
    ids = np.array([0, 10, 100, 1000, 10000], dtype=np.uint32)
    X, Y = dims[0], dims[1]
    pts = np.stack([ids % X, (ids // X) % Y, ids // (X * Y)], axis=1).astype(np.float32)
    m = _inserted(dims, pts)
    assert (m[ids] == (ids % X) | (((ids // X) % Y) << 10) | ((ids // (X * Y)) << 20)).all()
    assert (oracle.sqdist(m, dims, ids) == 0).all()
    d0 = oracle.dist(m, dims, ids)
    oracle.pba(m, dims)
    dn = oracle.dist(m, dims, ids + 1)
    assert (d0 == 0).all() and (dn != d0).all()


def test_distance_correctness_lattice_matches_exact():
    """distance_correctness (GV/test/testing_distance.cu:39-127): PBA(1,1,1) on the
    tie-rich equidistant lattice, 128x128x131, against an exact EDT; the
    reference's bar is max |sqrt difference| < 0.01 -- here it must be 0."""
    dims = (128, 128, 131)
    pts = refgeom.equidistant_points_fast(10_000, dims, 1.0)
    ins = _inserted(dims, pts)
    m = ins.copy()
    oracle.pba(m, dims)
    got = _sites_sqdist(m, dims)
    want = _exact_sqdist(ins, dims)
    assert np.array_equal(got, want)


# ---- literal launch order vs generalised sweeps -------------------------

@pytest.mark.parametrize("dims,seed,npts", [
    ((64, 64, 64), 0, 300),
    ((64, 64, 37), 1, 2000),
    ((32, 32, 100), 2, 50),
    ((48, 48, 16), 3, 5000),
])
def test_reference_order_equals_generalised(dims, seed, npts):
    rng = np.random.default_rng(seed)
    pts = (rng.random((npts, 3)) * np.asarray(dims)).astype(np.float32)
    a = _inserted(dims, pts)
    b = a.copy()
    oracle.pba_reference_order(a, dims)
    oracle.pba(b, dims)
    assert np.array_equal(a, b)


def test_reference_order_equals_generalised_lattice_and_edge_maps():
    dims = (64, 64, 40)
    cases = {
        "lattice": refgeom.equidistant_points_fast(100_000, dims, 1.0),
        "single": np.array([[10.5, 20.5, 30.5]], dtype=np.float32),
        "symmetric": np.array([[10.5, 32.5, 20.5], [53.5, 32.5, 20.5]], dtype=np.float32),
        "collinear": np.array([[5.5, 5.5, 5.5], [25.5, 25.5, 25.5], [45.5, 45.5, 35.5]], dtype=np.float32),
    }
    for name, pts in cases.items():
        a = _inserted(dims, pts)
        b = a.copy()
        oracle.pba_reference_order(a, dims)
        oracle.pba(b, dims)
        assert np.array_equal(a, b), name
    empty = oracle.dvm_empty(dims)
    e2 = empty.copy()
    oracle.pba(e2, dims)
    assert (e2 == DV_UNINIT).all()
    full = _inserted(dims, refgeom.box_of_points((0, 0, 0), (63.5, 63.5, 39.5), 1.0) + np.float32(0.25))
    assert (full != DV_UNINIT).all()
    f2 = full.copy()
    oracle.pba(f2, dims)
    assert np.array_equal(f2, full)


@pytest.mark.parametrize("dims,seed,npts", [
    ((17, 33, 9), 0, 40),
    ((96, 40, 70), 1, 500),
    ((1, 50, 50), 2, 20),
    ((50, 1, 50), 3, 20),
    ((50, 50, 1), 4, 20),
    ((70, 90, 65), 5, 3000),
])
def test_generalised_sqdist_is_exact(dims, seed, npts):
    rng = np.random.default_rng(seed)
    pts = (rng.random((npts, 3)) * np.asarray(dims)).astype(np.float32)
    ins = _inserted(dims, pts)
    m = ins.copy()
    oracle.pba(m, dims)
    assert np.array_equal(_sites_sqdist(m, dims), _exact_sqdist(ins, dims))


def test_bisector_restatement():
    # devicePBAintersection3DY: yM + (nx*(xM-x0) + nz*(zM-z0)) / ny
    assert oracle.isect(0, 0, 0, 0, 2, 0, 0, 0) == 1.0
    for args in [(3, 1, 7, 9, 4, 2, 5, 6), (1000, 3, 1022, 2, 1021, 0, 511, 7), (0, 0, 0, 1, 3, 1, 0, 0)]:
        x1, y1, z1, x2, y2, z2, x0, z0 = (np.float32(a) for a in args)
        xM, yM, zM = (np.float32((a + b) / np.float32(2)) for a, b in ((x1, x2), (y1, y2), (z1, z2)))
        want = np.float32(yM + np.float32(np.float32((x2 - x1) * (xM - x0) + (z2 - z1) * (zM - z0)) / (y2 - y1)))
        assert oracle.isect(*args) == want


# ---- collisions: known answers of GV/test/testing_voxelmap.cu / testing_voxellist.cu

def _bvm(dims, pts, meaning=1):
    m = oracle.bvm_empty(dims)
    oracle.bvm_insert(m, dims, 1.0, pts, meaning)
    return m


def test_collision_equidistant_counts_every_point():
    """collision (testing_voxelmap.cu:96-115): 10000 points, default dims 89x123x74."""
    dims = (89, 123, 74)
    pts = refgeom.equidistant_points_fast(10_000, dims, 1.0)
    a, b = _bvm(dims, pts), _bvm(dims, pts)
    assert oracle.bvm_collide(a, b) == 10_000


def test_collision_with_offset_8_18_18():
    """collision_with_offset (testing_voxelmap.cu:119-142)."""
    dims = (89, 123, 74)
    p1 = refgeom.box_of_points((2.1, 2.1, 2.1), (4.1, 4.1, 4.1), 0.5)
    p2 = refgeom.box_of_points((3.1, 3.1, 3.1), (5.1, 5.1, 5.1), 0.5)
    m1, m2 = _bvm(dims, p1), _bvm(dims, p2)
    lin = lambda o: o[2] * dims[0] * dims[1] + o[1] * dims[0] + o[0]
    assert oracle.bvm_collide(m1.copy(), m2) == 8
    assert oracle.bvm_collide(m1.copy(), m2, lin((-1, 0, -1))) == 18
    assert oracle.bvm_collide(m2.copy(), m1, lin((1, 0, 1))) == 18


def test_no_collision_checkerboard():
    """no_collision (testing_voxelmap.cu:144-168)."""
    dims = (89, 123, 74)
    black, white = refgeom.nonoverlapping_checkerboard(10_000, dims, 1.0)
    assert oracle.bvm_collide(_bvm(dims, black), _bvm(dims, white)) == 0


def _list_from_boxes(dims, meanings=(11, 12)):
    ids, vox = None, None
    boxes = [((1.1, 1.1, 1.1), (3.9, 3.9, 3.9)), ((2.1, 2.1, 2.1), (4.9, 4.9, 4.9))]
    for (lo, hi), mean in zip(boxes, meanings):
        ids, vox = oracle.list_insert(ids, vox, dims, 1.0, refgeom.box_of_points(lo, hi, 0.1), mean)
    return ids, vox


def test_list_vs_map_46_and_marks():
    """collide_bitvoxellist_with_prob_voxelmap / ..._bitvoxelmap (testing_voxellist.cu:111-238)."""
    dims = (89, 123, 74)
    ids, vox = _list_from_boxes(dims)
    assert ids.shape[0] == 46
    bmap = oracle.bvm_empty(dims)
    boxes = [((1.1, 1.1, 1.1), (3.9, 3.9, 3.9)), ((2.1, 2.1, 2.1), (4.9, 4.9, 4.9))]
    for lo, hi in boxes:
        oracle.bvm_insert(bmap, dims, 1.0, refgeom.box_of_points(lo, hi, 0.1), 1)
    v = vox.copy()
    assert oracle.list_collide_map(ids, v, bmap) == 46
    assert (v.reshape(-1, 32)[:, 0] & 4).all()  # every entry marked eBVM_COLLISION


def test_list_shifting_27_18_9_0():
    """collide_bitvoxellist_with_prob_voxelmap_shifting (testing_voxellist.cu:241-281)."""
    dims = (89, 123, 74)
    box = refgeom.box_of_points((1.1, 1.1, 1.1), (3.9, 3.9, 3.9), 0.1)
    ids, vox = oracle.list_insert(None, None, dims, 1.0, box, 1)
    bmap = _bvm(dims, box)
    for shift, want in [(0, 27), (0.5, 27), (1, 18), (1.5, 18), (2, 9), (2.5, 9), (3, 0), (3.5, 0)]:
        off = int(shift)  # Vector3i(shift, 0, 0) truncates
        assert oracle.list_collide_map(ids, vox.copy(), bmap, off) == want


def test_list_vs_list_46():
    """countingvoxellist_collide_bitvectorvoxellist (testing_voxellist.cu:692-738), bit-vector list form."""
    dims = (89, 123, 74)
    ids, _ = _list_from_boxes(dims)
    assert oracle.list_collide_list(ids, ids) == 46
    assert oracle.list_collide_list(ids[:10], ids[5:]) == 5


def _closed_form_phase1(occ: np.ndarray) -> np.ndarray:
    """The per-column closed form the occupancy-bit pass Z uses (edt.cu,
    pass_z_bits_item): between consecutive sites s1 < s2 of a column (s2 = 1023
    above the highest site, s1 = 1023 below the lowest), rows z <= (s1 + s2) >> 1
    take s1 and the others s2; with s1 = 1023 every row takes s2.  occ: bool
    [Z, Y, X]; returns the site z per voxel (1023 = none)."""
    Z = occ.shape[0]
    out = np.full(occ.shape, 1023, dtype=np.int64)
    for y in range(occ.shape[1]):
        for x in range(occ.shape[2]):
            sites = [int(z) for z in np.flatnonzero(occ[:, y, x])]
            for z in range(Z):
                below = [s for s in sites if s <= z]
                above = [s for s in sites if s > z]
                s1 = below[-1] if below else 1023
                s2 = above[0] if above else 1023
                if s1 == z:
                    out[z, y, x] = z
                elif s1 == 1023:
                    out[z, y, x] = s2
                else:
                    out[z, y, x] = s1 if z <= (s1 + s2) >> 1 else s2
    return out


@pytest.mark.parametrize("dims,density,seed", [((7, 5, 40), 0.05, 0), ((6, 4, 33), 0.3, 1), ((5, 5, 64), 0.01, 2),
                                               ((3, 2, 1), 0.5, 3)])
def test_closed_form_backward_flood_equals_phase1(dims, density, seed):
    """kernelPBAphase1FloodZ (GV/voxelmap/kernels/VoxelMapOperationsPBA.hpp:63-124)
    on an inserted map, restated by the oracle, equals the closed form above,
    ties (z equidistant from two sites) and the UNINIT-as-1023 arithmetic
    included."""
    X, Y, Z = dims
    rng = np.random.default_rng(seed)
    occ = rng.random((Z, Y, X)) < density
    occ[:, 0, 0] = False  # one empty column
    vmap = oracle.dvm_empty(dims)
    zz, yy, xx = np.nonzero(occ)
    vmap.reshape(Z, Y, X)[zz, yy, xx] = (xx | (yy << 10) | (zz << 20)).astype(np.uint32)
    oracle.phase1(vmap, dims)
    got = vmap.reshape(Z, Y, X)
    want_z = _closed_form_phase1(occ)
    gx = np.arange(X)[None, None, :]
    gy = np.arange(Y)[None, :, None]
    want = np.where(want_z == 1023, np.uint32(0x3FFFFFFF),
                    (gx | (gy << 10) | (want_z << 20)).astype(np.uint32))
    assert np.array_equal(got, want)
