"""GPU parity of voxelisation + EDT + discrete queries against the oracle
(bit-exact sites, so squared distances and tie-breaking match)."""
import numpy as np
import pytest
import torch

import gvx
import oracle
import refgeom
from gpu_helpers import first_mismatch, gpu_edt, oracle_edt, to_u32
import workloads

pytestmark = pytest.mark.gpu


def _check(dims, side, pts):
    ins_o, edt_o = oracle_edt(dims, side, pts)
    ins_g, edt_g, dvm = gpu_edt(dims, side, pts)
    assert np.array_equal(ins_g, ins_o), first_mismatch(ins_g, ins_o, dims)
    assert np.array_equal(edt_g, edt_o), first_mismatch(edt_g, edt_o, dims)
    return dvm, edt_o


@pytest.mark.parametrize("dims,seed,npts", [
    ((64, 64, 64), 0, 300),
    ((128, 128, 131), 1, 5000),
    ((32, 32, 32), 2, 1),
    ((17, 33, 9), 3, 40),
    ((96, 40, 70), 4, 500),
    ((1, 50, 50), 5, 20),
    ((50, 1, 50), 6, 20),
    ((50, 50, 1), 7, 20),
    ((33, 65, 129), 8, 2000),
    ((255, 3, 7), 9, 30),
    ((200, 200, 20), 10, 20000),
])
def test_edt_random_scenes(dims, seed, npts):
    rng = np.random.default_rng(seed)
    pts = (rng.random((npts, 3)) * np.asarray(dims)).astype(np.float32)
    _check(dims, 1.0, pts)


@pytest.mark.parametrize("dims", [(96, 40, 70), (33, 65, 129), (256, 256, 64), (1, 50, 50), (50, 1, 50), (7, 9, 3)])
def test_fused_yx_sweep_equals_separate_passes(dims):
    """The fused y -> x launch (stage 3, what parallelBanding3D runs) gives the
    same map as the y and x sweeps launched one after the other, and its
    bounded slice waits all end in time."""
    rng = np.random.default_rng(sum(dims))
    n = max(1, int(np.prod(dims)) // 200)
    pts = torch.as_tensor((rng.random((n, 3)) * np.asarray(dims)).astype(np.float32)).cuda()
    a = gvx.DistanceVoxelMap(dims, 1.0)
    b = gvx.DistanceVoxelMap(dims, 1.0)
    for m in (a, b):
        m.insertPointCloud(pts)
        m.edt_pass(0)
    a.edt_pass(1)
    a.edt_pass(2)
    b.edt_pass(3)
    assert b.edt_check() == 0
    assert torch.equal(a.data(), b.data())


def test_edt_tie_rich_lattice():
    dims = (128, 128, 131)
    _check(dims, 1.0, refgeom.equidistant_points_fast(10_000, dims, 1.0))


def test_edt_special_maps():
    dims = (64, 64, 40)
    for pts in [np.zeros((0, 3), np.float32),
                np.array([[10.5, 20.5, 30.5]], np.float32),
                np.array([[10.5, 32.5, 20.5], [53.5, 32.5, 20.5]], np.float32),
                np.array([[5.5, 5.5, 5.5], [25.5, 25.5, 25.5], [45.5, 45.5, 35.5]], np.float32),
                refgeom.box_of_points((0, 0, 0), (63.5, 63.5, 39.5), 1.0) + np.float32(0.25)]:
        _check(dims, 1.0, pts)


def test_edt_negative_nan_and_outside_points():
    dims = (40, 40, 40)
    rng = np.random.default_rng(3)
    pts = (rng.random((500, 3)) * 50 - 5).astype(np.float32)  # some negative, some beyond the map
    pts[:7] = np.nan
    dvm, _ = _check(dims, 1.0, pts)
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    dvm.clearMap()
    dvm.insertPointCloud(torch.as_tensor(pts), outside=flag)
    assert int(flag.item()) == 1


def test_edt_c1_config():
    sc = workloads.c1_scene()
    dvm, edt_o = _check(sc.dims, sc.side, sc.points)
    ids = workloads.c1_queries()
    got = dvm.getSquaredDistances(torch.as_tensor(ids.astype(np.int64))).cpu().numpy()
    assert np.array_equal(got, oracle.sqdist(edt_o, sc.dims, ids))
    got = dvm.getDistances(torch.as_tensor(ids.astype(np.int64))).cpu().numpy()
    assert np.array_equal(got, oracle.dist(edt_o, sc.dims, ids))
    got = to_u32(dvm.gatherVoxelsByIndex(torch.as_tensor(ids.astype(np.int64))))
    assert np.array_equal(got, edt_o[ids])
    assert np.array_equal(dvm.squaredDistanceMap().cpu().numpy(), oracle.sqdist_map(edt_o, sc.dims))


def test_edt_256_scene_and_repeat_is_deterministic():
    sc = workloads.c3_scene()
    dvm, edt_o = _check(sc.dims, sc.side, sc.points)
    dvm.clearMap()
    dvm.insertPointCloud(torch.as_tensor(sc.points))
    dvm.parallelBanding3D()
    assert np.array_equal(to_u32(dvm.data()), edt_o)


def test_edt_twice_matches_oracle_on_already_transformed_map():
    """Running the EDT on an EDT'd map (a legal reference call sequence)."""
    dims = (48, 48, 48)
    rng = np.random.default_rng(11)
    pts = (rng.random((300, 3)) * 48).astype(np.float32)
    _, edt_o = oracle_edt(dims, 1.0, pts)
    again_o = edt_o.copy()
    oracle.pba(again_o, dims)
    _, _, dvm = gpu_edt(dims, 1.0, pts)
    dvm.parallelBanding3D()
    assert np.array_equal(to_u32(dvm.data()), again_o)


def test_edt_c2_512_sqdist_matches_exact_property():
    """512^3 C2 scene: full bit-exact comparison with the oracle."""
    pts = workloads.c2_points()
    dims, side = (512, 512, 512), 0.005
    ins_o, edt_o = oracle_edt(dims, side, pts)
    ins_g, edt_g, dvm = gpu_edt(dims, side, pts)
    assert np.array_equal(ins_g, ins_o), first_mismatch(ins_g, ins_o, dims)
    assert np.array_equal(edt_g, edt_o), first_mismatch(edt_g, edt_o, dims)


def test_sqdist_out_of_range_ids_are_guarded():
    dims = (16, 16, 16)
    _, _, dvm = gpu_edt(dims, 1.0, np.array([[1.5, 1.5, 1.5]], np.float32))
    ids = torch.tensor([0, 16 ** 3 - 1, 16 ** 3, 2 ** 31], dtype=torch.int64)
    out = dvm.getSquaredDistances(ids).cpu().numpy()
    assert out[0] == 3 and out[2] == 2147483647 and out[3] == 2147483647


def _walls(dims, seed):
    """Points on planes parallel to z: many columns hold more sites than pass
    Z's on-chip ring, plus scattered points."""
    rng = np.random.default_rng(seed)
    X, Y, Z = dims
    pts = [np.stack([np.full(Z, 3.5), np.full(Z, 5.5), np.arange(Z) + 0.5], 1)]
    for _ in range(4):
        x = rng.integers(0, X)
        ys, zs = np.meshgrid(np.arange(rng.integers(0, Y // 2), Y), np.arange(Z // 3, Z), indexing="ij")
        pts.append(np.stack([np.full(ys.size, x + 0.5), ys.ravel() + 0.5, zs.ravel() + 0.5], 1))
    pts.append(rng.random((500, 3)) * np.asarray(dims))
    return np.concatenate(pts).astype(np.float32)


@pytest.mark.parametrize("dims", [(70, 40, 90), (64, 64, 200), (33, 17, 1023)])
def test_edt_dense_columns(dims):
    _check(dims, 1.0, _walls(dims, sum(dims)))


@pytest.mark.parametrize("case", ["random", "walls", "c1", "outside", "tall_sparse", "few", "empty"])
def test_voxelize_edt_equals_clear_insert_edt(case):
    dims = {"random": (96, 40, 70), "walls": (70, 40, 90), "c1": (128, 128, 128), "outside": (40, 44, 48),
            "tall_sparse": (40, 36, 700), "few": (33, 40, 320), "empty": (32, 32, 96)}[case]
    if case in ("random", "tall_sparse", "few", "empty"):
        # tall_sparse and few: mostly site-free 32-row z chunks, sites below and
        # above them, and (Z > 512) rows the reference leaves uninitialised
        n = {"random": 3000, "tall_sparse": 300, "few": 6, "empty": 0}[case]
        pts = (np.random.default_rng(1).random((n, 3)) * np.asarray(dims)).astype(np.float32).reshape(n, 3)
        side = 1.0
    elif case == "walls":
        pts, side = _walls(dims, 3), 1.0
    elif case == "c1":
        sc = workloads.c1_scene()
        pts, side = sc.points, sc.side
    else:  # negative, NaN and beyond-the-map coordinates: the outside flag and voxel 0
        rng = np.random.default_rng(2)
        pts = (rng.random((400, 3)) * 1.4 - 0.2) * np.asarray(dims)
        pts[:5] = np.nan
        pts = pts.astype(np.float32)
        side = 1.0
    _, want = oracle_edt(dims, side, pts)
    p = torch.as_tensor(pts).cuda()
    a = gvx.DistanceVoxelMap(dims, side)
    b = gvx.DistanceVoxelMap(dims, side)
    fa = torch.zeros(1, dtype=torch.int32, device="cuda")
    fb = torch.zeros(1, dtype=torch.int32, device="cuda")
    a.clearMap()
    a.insertPointCloud(p, outside=fa)
    a.parallelBanding3D()
    b.insertPointCloud(torch.as_tensor(np.random.default_rng(9).random((100, 3)) * np.asarray(dims) * side,
                                       dtype=torch.float32).cuda())
    b.parallelBanding3D()  # stale content that the fused call must not depend on
    b.voxelize_edt(p, outside=fb)
    assert b.edt_check() == 0
    assert torch.equal(a.data(), b.data())
    assert int(fa.item()) == int(fb.item())
    assert np.array_equal(to_u32(b.data()), want)


def test_bisector_quotient_equals_ieee_divide_over_domain():
    """The sweeps round the bisector quotient without the general divide; every
    (numerator, divisor) they can meet gives the IEEE divide's bits."""
    import ctypes
    from gvx import _abi
    bad = ctypes.c_uint64(1)
    _abi.check(_abi.lib().gvx_check_bisector_quotient(ctypes.byref(bad)))
    assert bad.value == 0


@pytest.mark.parametrize("dims", [(1, 40, 60), (5, 3, 100), (33, 1, 20), (70, 9, 2), (1, 1, 300), (31, 33, 17)])
def test_thin_maps_every_sweep_configuration(dims):
    """x or y below 32: sweep items span z slices (several slice counters per
    item in the fused launch); every configuration and voxelize_edt agree with
    the oracle."""
    rng = np.random.default_rng(sum(dims))
    pts = (rng.random((max(1, int(np.prod(dims)) // 50), 3)) * np.asarray(dims)).astype(np.float32)
    _, want = oracle_edt(dims, 1.0, pts)
    p = torch.as_tensor(pts).cuda()
    m = gvx.DistanceVoxelMap(dims, 1.0)
    for rows in (16, 32):
        for fused in (0, 1):
            m.set_edt_config(rows=rows, fused=fused)
            m.clearMap()
            m.insertPointCloud(p)
            m.parallelBanding3D()
            assert m.edt_check() == 0
            assert np.array_equal(to_u32(m.data()), want), (rows, fused)
            m.voxelize_edt(p)
            assert m.edt_check() == 0
            assert np.array_equal(to_u32(m.data()), want), ("voxelize", rows, fused)


@pytest.mark.parametrize("dims,npts", [((1023, 40, 3), 30), ((1023, 40, 3), 20000), ((7, 1023, 5), 40),
                                       ((1023, 1023, 1), 300)])
def test_longest_rows(dims, npts):
    """Rows of 1023 voxels along x or y: stacks up to 1023 entries deep and the
    largest bisector divisors (2046), sparse and dense, fused and separate."""
    rng = np.random.default_rng(npts)
    pts = (rng.random((npts, 3)) * np.asarray(dims)).astype(np.float32)
    _, want = oracle_edt(dims, 1.0, pts)
    p = torch.as_tensor(pts).cuda()
    m = gvx.DistanceVoxelMap(dims, 1.0)
    for fused in (1, 0):
        m.set_edt_config(rows=16, fused=fused)
        m.voxelize_edt(p)
        assert m.edt_check() == 0
        assert np.array_equal(to_u32(m.data()), want), fused


@pytest.mark.parametrize("dims", [(64, 40, 70), (37, 29, 33), (5, 3, 40)])
@pytest.mark.parametrize("where", ["first", "middle", "last"])
def test_filled_map_with_one_moved_site_takes_the_general_pass(dims, where):
    """parallelBanding3D on an inserted map reads occupancy bits when every
    voxel is UNINIT or its own site; one voxel holding another voxel's
    coordinates must send pass Z down the general path, bit-exact."""
    rng = np.random.default_rng(len(where) + dims[0])
    pts = (rng.random((300, 3)) * np.asarray(dims)).astype(np.float32)
    ins = oracle.dvm_empty(dims)
    oracle.dvm_insert(ins, dims, 1.0, pts)
    n = int(np.prod(dims))
    idx = {"first": 0, "middle": n // 2 + 7, "last": n - 1}[where]
    ins[idx] = np.uint32(3 | (1 << 10) | (2 << 20))  # the site (3, 1, 2), not this voxel's own
    want = ins.copy()
    oracle.pba(want, dims)
    m = gvx.DistanceVoxelMap(dims, 1.0)
    m.data().copy_(torch.as_tensor(ins.view(np.int32)).cuda())
    m.parallelBanding3D()
    assert m.edt_check() == 0
    assert np.array_equal(to_u32(m.data()), want), first_mismatch(to_u32(m.data()), want, dims)
    # and the plain inserted map (no moved site) still matches through the bits path
    m.clearMap()
    m.insertPointCloud(torch.as_tensor(pts).cuda())
    m.parallelBanding3D()
    _, want2 = oracle_edt(dims, 1.0, pts)
    assert np.array_equal(to_u32(m.data()), want2)
