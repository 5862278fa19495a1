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

# Tolerances (voxel units for distances, dimensionless for gradients).
DIST_MAX_ERR_VOX = 1e-5
GRAD_MAX_ERR = 1e-4


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
    assert err.max() <= 1e-3


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


def test_traj_cost_and_adjoint(scene):
    sc, edt, dvm = scene
    spec = workloads.arm_spec()
    arm = gvx.make_arm(spec)
    q = workloads.c4_trajectories(16, 64)
    margin = 0.05
    cost = dvm.traj_cost(arm, torch.as_tensor(q), margin).cpu().numpy().astype(np.float64)
    want = oracle.traj_cost64(edt, sc.dims, sc.side, spec, q, margin)
    assert np.allclose(cost, want, rtol=1e-4, atol=1e-4), (cost, want)
    gcost = np.linspace(0.5, 1.5, q.shape[0]).astype(np.float32)
    gq = dvm.traj_cost_backward(arm, torch.as_tensor(q), margin, torch.as_tensor(gcost)).cpu().numpy()
    # FP64 central differences on a subset of waypoints/joints
    h = 1e-4
    rng = np.random.default_rng(0)
    errs = []
    for _ in range(60):
        b, w, j = rng.integers(0, q.shape[0]), rng.integers(0, q.shape[1]), rng.integers(0, q.shape[2])
        qp = q[b:b + 1].astype(np.float64).copy()
        qm = qp.copy()
        qp[0, w, j] += h
        qm[0, w, j] -= h
        fd = gcost[b] * (oracle.traj_cost64(edt, sc.dims, sc.side, spec, qp, margin)[0]
                         - oracle.traj_cost64(edt, sc.dims, sc.side, spec, qm, margin)[0]) / (2 * h)
        errs.append(abs(fd - gq[b, w, j]) / max(1e-3, abs(fd)))
    errs = np.asarray(errs)
    print(f"\ntrajectory adjoint vs FP64 central differences: median rel err {np.median(errs):.2e}, "
          f"90th pct {np.percentile(errs, 90):.2e}")
    assert np.median(errs) < 1e-2


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
