"""GPU checks of the continuous queries against the FP64 oracle:
trilinear distance + gradient (and its adjoint), sphere clearance, the hinge
trajectory cost and its adjoint (FP64 central differences)."""
import numpy as np
import pytest
import torch

import gvx
import oracle
from gpu_helpers import gpu_edt, to_u32
import workloads

pytestmark = pytest.mark.gpu

# Tolerances: the FP32 queries against FP64 restatements of the same
# interpolant, 1e-5 in voxel units for distances and 1e-5 for the
# dimensionless spatial gradient d(distance)/d(position).
DIST_MAX_ERR_VOX = 1e-5
GRAD_MAX_ERR = 1e-5


@pytest.fixture(scope="module")
def scene():
    sc = workloads.c3_scene()
    _, edt, dvm = gpu_edt(sc.dims, sc.side, sc.points)
    return sc, edt, dvm


def _near_face(u_frac, h_vox):
    return np.any((u_frac < h_vox) | (u_frac > 1 - h_vox), axis=1)


def test_trilinear_matches_fp64(scene):
    sc, edt, dvm = scene
    pts = workloads.c4_points(200_000, sc.dims, sc.side)
    d32, g32 = dvm.trilinear(torch.as_tensor(pts))
    d64, g64 = oracle.trilinear64(edt, sc.dims, sc.side, pts)
    err_vox = np.abs(d32.cpu().numpy().astype(np.float64) - d64) / sc.side
    # the gradient jumps across cell faces: compare away from them (where the
    # FP64 cell choice itself is decided by the last bit)
    u = pts.astype(np.float64) / np.float64(np.float32(sc.side)) - 0.5
    on_face = _near_face(u - np.floor(u), 1e-6)
    gerr = np.abs(g32.cpu().numpy().astype(np.float64) - g64)[~on_face]
    print(f"\ntrilinear FP32 vs FP64: max {err_vox.max():.3e} vox, rms {np.sqrt((err_vox**2).mean()):.3e} vox; "
          f"grad max {gerr.max():.3e} rms {np.sqrt((gerr**2).mean()):.3e} ({int(on_face.sum())} pts on faces skipped)")
    assert err_vox.max() <= DIST_MAX_ERR_VOX
    assert gerr.max() <= GRAD_MAX_ERR


def test_trilinear_gradient_matches_central_differences(scene):
    sc, edt, dvm = scene
    pts = workloads.c4_points(20_000, sc.dims, sc.side).astype(np.float64)
    h = 1e-4
    u = pts / sc.side - 0.5
    keep = ~_near_face(u - np.floor(u), 1.5 * h / sc.side)
    pts = pts[keep]
    fd = np.zeros_like(pts)
    for a in range(3):
        e = np.zeros(3)
        e[a] = h
        dp, _ = oracle.trilinear64(edt, sc.dims, sc.side, pts + e)
        dm, _ = oracle.trilinear64(edt, sc.dims, sc.side, pts - e)
        fd[:, a] = (dp - dm) / (2 * h)
    _, g32 = dvm.trilinear(torch.as_tensor(pts.astype(np.float32)))
    err = np.abs(g32.cpu().numpy() - fd)
    print(f"\ngradient vs FP64 central differences (h=1e-4 m, {pts.shape[0]} pts off cell faces): max {err.max():.3e}")
    # Inside one cell the interpolant is linear along each axis, so the
    # central difference is exact up to FP64 rounding (eps * d / h ~ 1e-11):
    # the bound is the FP32 gradient's own tolerance.
    assert err.max() <= GRAD_MAX_ERR


def test_trilinear_adjoint_is_grad_times_upstream(scene):
    sc, edt, dvm = scene
    pts = torch.as_tensor(workloads.c4_points(50_000, sc.dims, sc.side))
    _, g = dvm.trilinear(pts)
    gout = torch.randn(pts.shape[0], device="cuda")
    gx = dvm.trilinear_backward(pts, gout)
    assert torch.equal(gx, g * gout[:, None])


def test_trilinear_clamps_outside_points(scene):
    sc, edt, dvm = scene
    pts = np.array([[-1.0, 1.0, 1.0], [10.0, 1.0, 1.0], [1.0, 1.0, np.nan], [0.005, 0.005, 0.005]], np.float32)
    d32, g32 = dvm.trilinear(torch.as_tensor(pts))
    d64, g64 = oracle.trilinear64(edt, sc.dims, sc.side, pts)
    assert np.allclose(d32.cpu().numpy(), d64, atol=1e-6)
    assert np.allclose(g32.cpu().numpy(), g64, atol=1e-5)
    assert g32[0, 0].item() == 0.0 and g32[1, 0].item() == 0.0


def test_sphere_clearance_matches_fp64(scene):
    sc, edt, dvm = scene
    spec = workloads.arm_spec()
    arm = gvx.make_arm(spec)
    q = workloads.c3_configs(512)
    got = dvm.sphere_clearance(arm, torch.as_tensor(q)).cpu().numpy().astype(np.float64)
    want = oracle.sphere_clearance64(edt, sc.dims, sc.side, spec, q)
    err = np.abs(got - want) / sc.side
    print(f"\nsphere clearance FP32 vs FP64: max {err.max():.3e} vox, rms {np.sqrt((err**2).mean()):.3e} vox")
    # FP64 forward kinematics, and the centre split into cell and fraction in
    # FP64: only the fraction and the query's own arithmetic round to FP32
    assert err.max() < 1e-5


def _traj_case(n_traj=16, n_wp=64):
    spec = workloads.arm_spec()
    q = workloads.c4_trajectories(n_traj, n_wp)
    gcost = np.linspace(0.5, 1.5, n_traj).astype(np.float32)
    return spec, q, gcost, 0.05


def test_traj_cost_matches_fp64(scene):
    sc, edt, dvm = scene
    spec, q, _, margin = _traj_case()
    arm = gvx.make_arm(spec)
    cost = dvm.traj_cost(arm, torch.as_tensor(q), margin).cpu().numpy().astype(np.float64)
    want = oracle.traj_cost64(edt, sc.dims, sc.side, spec, q, margin)
    _, _, gap = oracle.traj_cost_grad64(edt, sc.dims, sc.side, spec, q, margin, np.ones(q.shape[0]))
    c = oracle.sphere_centres64(spec, q)
    d, _ = oracle.trilinear64(edt, sc.dims, sc.side, c.reshape(-1, 3))
    r = np.asarray(spec["r"], np.float32).astype(np.float64)
    n_active = ((np.float32(margin) - (d.reshape(c.shape[:-1]) - r)) > 0).sum(axis=(1, 2))
    err = np.abs(cost - want)
    # Each active hinge term carries the distance query's error (<= 1e-5
    # voxel = 1e-5 * side metres); summing n positive float terms adds at
    # most n * 2^-23 of the sum.  Trajectories with a waypoint whose active
    # set a rounding could flip (a clearance within 1e-6 m of the margin) are
    # left out.
    ok = gap.min(axis=1) > 1e-6
    assert ok.mean() > 0.8
    bound = 1e-5 * sc.side * n_active + n_active * 2.0 ** -23 * want
    print(f"\ntrajectory cost FP32 vs FP64: max {err[ok].max():.3e} m, "
          f"max err/bound {(err / np.maximum(bound, 1e-30))[ok].max():.3f}")
    assert n_active.sum() > 0
    assert np.all(err[ok] <= bound[ok] + 1e-12)


def test_traj_adjoint_matches_fp64_analytic_and_central_differences(scene):
    sc, edt, dvm = scene
    spec, q, gcost, margin = _traj_case()
    arm = gvx.make_arm(spec)
    gq = dvm.traj_cost_backward(arm, torch.as_tensor(q), margin, torch.as_tensor(gcost)).cpu().numpy().astype(np.float64)
    want, scale, gap = oracle.traj_cost_grad64(edt, sc.dims, sc.side, spec, q, margin, gcost)
    ok = (gap > 1e-6)[..., None] & np.ones_like(want, dtype=bool)  # no active-set flip possible
    assert ok.mean() > 0.99
    # The adjoint multiplies each active sphere's spatial gradient (component
    # error <= GRAD_MAX_ERR) with its moment arm z_k x (c_s - o_k) and sums in
    # FP64: its error is at most GRAD_MAX_ERR times the summed |arm|_1
    # (`scale`), plus the final rounding to float.
    err = np.abs(gq - want)
    bound = GRAD_MAX_ERR * scale + 2.0 ** -23 * np.abs(want)
    ratio = (err / np.maximum(bound, 1e-30))[ok]
    print(f"\ntrajectory adjoint vs FP64 analytic: max err {err[ok].max():.3e}, max err/bound {ratio.max():.3f}, "
          f"rms err/scale {np.sqrt(np.mean((err[ok] / np.maximum(scale[ok], 1e-30)) ** 2)):.2e}")
    assert np.all(err[ok] <= bound[ok] + 1e-12)
    assert np.abs(want).max() > 0
    # The FP64 analytic adjoint against FP64 central differences, h = 1e-5
    # rad: inside one cell and with a fixed active set the cost is smooth in q
    # and the truncation error is ~h^2 (measured below 1e-8 of `scale`);
    # samples whose +-h step moves a sphere across a cell face (where the
    # trilinear gradient jumps) or flips a hinge are skipped.
    h = 1e-5
    side = float(np.float32(sc.side))
    r = np.asarray(spec["r"], np.float32).astype(np.float64)

    def state(qw):
        c = oracle.sphere_centres64(spec, qw)
        d, _ = oracle.trilinear64(edt, sc.dims, sc.side, c.reshape(-1, 3))
        return np.floor(c / side - 0.5), (np.float32(margin) - (d.reshape(c.shape[:-1]) - r)) > 0

    rng = np.random.default_rng(0)
    checked = 0
    for _ in range(80):
        b, w, j = rng.integers(0, q.shape[0]), rng.integers(0, q.shape[1]), rng.integers(0, q.shape[2])
        qp = q[b:b + 1].astype(np.float64).copy()
        qm = qp.copy()
        qp[0, w, j] += h
        qm[0, w, j] -= h
        cp, ap = state(qp[:, w])
        cm, am = state(qm[:, w])
        if not (np.array_equal(cp, cm) and np.array_equal(ap, am)):
            continue
        fd = gcost[b] * (oracle.traj_cost64(edt, sc.dims, sc.side, spec, qp, margin)[0]
                         - oracle.traj_cost64(edt, sc.dims, sc.side, spec, qm, margin)[0]) / (2 * h)
        assert abs(fd - want[b, w, j]) <= 1e-7 * scale[b, w, j] + 1e-9, (b, w, j, fd, want[b, w, j])
        assert abs(fd - gq[b, w, j]) <= bound[b, w, j] + 1e-7 * scale[b, w, j] + 1e-9, (b, w, j)
        checked += 1
    assert checked >= 60


def test_torch_autograd_functions(scene):
    """libtorch torch::autograd::Function wrappers: backward = the adjoint kernels."""
    from gvx import autograd

    sc, edt, dvm = scene
    pts = torch.as_tensor(workloads.c4_points(10_000, sc.dims, sc.side)).cuda().requires_grad_(True)
    d = autograd.trilinear_distance(pts, dvm)
    w = torch.linspace(0.5, 2.0, d.shape[0], device="cuda")
    (d * w).sum().backward()
    _, g = dvm.trilinear(pts.detach())
    assert torch.allclose(pts.grad, g * w[:, None], atol=0, rtol=0)
    assert torch.equal(d.detach(), dvm.trilinear(pts.detach(), with_grad=False))

    spec = workloads.arm_spec()
    arm = gvx.make_arm(spec)
    q0 = torch.as_tensor(workloads.c3_configs(8)).cuda().requires_grad_(True)
    q1 = torch.as_tensor(workloads.c3_configs(16)[8:]).cuda()
    t = torch.linspace(0, 1, 32, device="cuda")[None, :, None]
    q = q0[:, None, :] + (q1 - q0)[:, None, :] * t          # [8, 32, 7] waypoints
    cost = autograd.trajectory_cost(q, dvm, arm, 0.05)
    cost.sum().backward()
    gq = dvm.traj_cost_backward(arm, q.detach(), 0.05, torch.ones(8, device="cuda"))
    want = (gq * (1 - t)).sum(1)                               # chain rule through the interpolation
    assert torch.allclose(q0.grad, want, rtol=1e-5, atol=1e-6)


def test_trilinear_corner_pair_paths(scene):
    """Corner pairs along x are read with one 16-byte load when both lie in one
    aligned word inside the map, one at a time otherwise (the pair straddles a
    word, the word would pass the map's end, or the axis is one voxel wide).
    Every path gives the FP64 oracle's values: the map's last cells, cells at
    each x mod 4, and a map one voxel wide in x."""
    sc, edt, dvm = scene
    rng = np.random.default_rng(3)
    hi = (np.asarray(sc.dims) - 0.5) * sc.side
    edge = hi - rng.random((4000, 3)) * 1.5 * sc.side  # the last cells
    cells = rng.integers(0, np.asarray(sc.dims) - 1, size=(4000, 3))
    cells[:, 0] = (cells[:, 0] & ~3) + np.arange(4000) % 4  # i0 at every x mod 4
    inner = (cells + 0.5 + rng.random((4000, 3))) * sc.side
    pts = np.concatenate([edge, np.minimum(inner, hi)]).astype(np.float32)
    d32, g32 = dvm.trilinear(torch.as_tensor(pts))
    d64, g64 = oracle.trilinear64(edt, sc.dims, sc.side, pts)
    assert np.abs(d32.cpu().numpy().astype(np.float64) - d64).max() / sc.side <= DIST_MAX_ERR_VOX
    u = pts.astype(np.float64) / np.float64(np.float32(sc.side)) - 0.5
    off = ~_near_face(u - np.floor(u), 1e-6)
    assert np.abs(g32.cpu().numpy().astype(np.float64) - g64)[off].max() <= GRAD_MAX_ERR
    thin = (1, 40, 30)
    tp = (rng.random((200, 3)) * thin).astype(np.float32)
    _, tedt, tdvm = gpu_edt(thin, 1.0, tp)
    q = (rng.random((3000, 3)) * thin).astype(np.float32)
    td32, _ = tdvm.trilinear(torch.as_tensor(q))
    td64, _ = oracle.trilinear64(tedt, thin, 1.0, q)
    assert np.abs(td32.cpu().numpy().astype(np.float64) - td64).max() <= DIST_MAX_ERR_VOX
