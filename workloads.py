"""Seeded synthetic workloads (numpy PCG64) for the five benchmark configs.

C1  128^3 @ 1 cm: 40 random boxes (surface samples) + 5% outliers, 50k points;
    100k uniform voxel-id queries.
C2  512^3 @ 5 mm: floor plane + 25 boxes seen by 4 ray-cast 640x480 depth
    images (pinhole fx=fy=525, cx=319.5, cy=239.5, sigma 2 mm), back-projected
    (~1.2M points); a second map of 64 random capsules sampled at side/2.
C3  256^3 @ 1 cm scene (C1 generator scaled to 2.56 m); synthetic 7-DOF DH arm
    with 56 spheres, 4096 configurations; 4096 voxel lists of log-uniform
    length in [2k, 200k].
C4  256^3 map as C3; 1M uniform points inside the voxel-centre lattice;
    512 trajectories x 64 waypoints.
C5  64 maps with dims log-uniform in [64, 384] per axis, each with its own
    box scene of 10k..1M points.

No public dataset is involved; the reference ships none for this path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


# ---------------------------------------------------------------------------
# box scenes
# ---------------------------------------------------------------------------

def _split_counts(total: int, weights: np.ndarray) -> np.ndarray:
    w = np.asarray(weights, dtype=np.float64)
    raw = total * w / w.sum()
    c = np.floor(raw).astype(np.int64)
    rem = total - int(c.sum())
    if rem > 0:
        order = np.argsort(-(raw - c), kind="stable")
        c[order[:rem]] += 1
    return c


def box_surface_points(rng: np.random.Generator, lo: np.ndarray, hi: np.ndarray, n: int) -> np.ndarray:
    """n points uniform on the surface of the AABB [lo, hi]."""
    e = hi - lo
    areas = np.array([e[1] * e[2], e[1] * e[2], e[0] * e[2], e[0] * e[2], e[0] * e[1], e[0] * e[1]])
    counts = _split_counts(n, areas)
    out = []
    for f, c in enumerate(counts):
        if c == 0:
            continue
        p = lo + rng.random((c, 3)) * e
        axis, side = f // 2, f % 2
        p[:, axis] = hi[axis] if side else lo[axis]
        out.append(p)
    return np.concatenate(out, axis=0) if out else np.zeros((0, 3))


def box_scene(seed: int, extent: np.ndarray, n_boxes: int = 40, n_points: int = 50_000, outlier_frac: float = 0.05,
              edge_range=(0.05, 0.30)) -> np.ndarray:
    """Surfaces of n_boxes random AABBs (edge per axis uniform in edge_range,
    scaled with the extent relative to 1.28 m) plus uniform outliers."""
    rng = np.random.default_rng(seed)
    extent = np.asarray(extent, dtype=np.float64)
    scale = extent / 1.28
    n_out = int(round(n_points * outlier_frac))
    n_surf = n_points - n_out
    edges = rng.uniform(edge_range[0], edge_range[1], size=(n_boxes, 3)) * scale
    edges = np.minimum(edges, extent * 0.999)
    lo = rng.random((n_boxes, 3)) * (extent - edges)
    hi = lo + edges
    areas = 2 * (edges[:, 0] * edges[:, 1] + edges[:, 1] * edges[:, 2] + edges[:, 0] * edges[:, 2])
    counts = _split_counts(n_surf, areas)
    pts = [box_surface_points(rng, lo[b], hi[b], int(counts[b])) for b in range(n_boxes)]
    pts.append(rng.random((n_out, 3)) * extent)
    return np.concatenate(pts, axis=0).astype(np.float32)


# ---------------------------------------------------------------------------
# C1
# ---------------------------------------------------------------------------

@dataclass
class MapScene:
    dims: tuple
    side: float
    points: np.ndarray


def c1_scene() -> MapScene:
    return MapScene((128, 128, 128), 0.01, box_scene(0, np.array([1.28, 1.28, 1.28])))


def c1_queries(n: int = 100_000) -> np.ndarray:
    return np.random.default_rng(1).integers(0, 128 ** 3, size=n, dtype=np.int64).astype(np.uint32)


# ---------------------------------------------------------------------------
# C2: depth images of a floor + boxes, and a capsule map
# ---------------------------------------------------------------------------

def _look_at(eye: np.ndarray, target: np.ndarray) -> np.ndarray:
    """Camera-to-world rotation: z forward, x right, y down."""
    z = target - eye
    z = z / np.linalg.norm(z)
    up = np.array([0.0, 0.0, 1.0])
    x = np.cross(z, up)
    x = x / np.linalg.norm(x)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1)


def _ray_aabb(o: np.ndarray, d: np.ndarray, lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """Entry parameter of rays o + t d into [lo, hi] (inf when missed)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / d
        t0 = (lo - o) * inv
        t1 = (hi - o) * inv
    tmin = np.nanmax(np.minimum(t0, t1), axis=1)
    tmax = np.nanmin(np.maximum(t0, t1), axis=1)
    hit = (tmax >= tmin) & (tmax > 0)
    return np.where(hit, np.maximum(tmin, 0.0), np.inf)


def c2_points(width: int = 640, height: int = 480, n_cams: int = 4) -> np.ndarray:
    extent = 2.56
    floor_z = 0.10
    rng = np.random.default_rng(0)
    nb = 25
    edges = rng.uniform(0.05, 0.5, size=(nb, 3))
    lo = np.empty((nb, 3))
    lo[:, :2] = rng.random((nb, 2)) * (extent - edges[:, :2])
    lo[:, 2] = floor_z
    hi = lo + edges
    noise = np.random.default_rng(2)
    fx = fy = 525.0
    cx, cy = 319.5, 239.5
    u, v = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64))
    dc = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u)], axis=-1).reshape(-1, 3)
    target = np.array([extent / 2, extent / 2, floor_z])
    clouds = []
    for k in range(n_cams):
        phi = 2 * math.pi * k / n_cams + math.pi / 4
        eye = np.array([extent / 2 + 1.2 * math.cos(phi), extent / 2 + 1.2 * math.sin(phi), 1.5])
        R = _look_at(eye, target)
        d = dc @ R.T  # world direction, camera-z component 1 => t == depth
        o = np.broadcast_to(eye, d.shape)
        with np.errstate(divide="ignore", invalid="ignore"):
            t = np.where(d[:, 2] < 0, (floor_z - eye[2]) / d[:, 2], np.inf)
        for b in range(nb):
            t = np.minimum(t, _ray_aabb(o, d, lo[b], hi[b]))
        ok = np.isfinite(t)
        z = t[ok] + noise.normal(0.0, 0.002, size=int(ok.sum()))
        pc = dc[ok] * z[:, None]
        clouds.append(pc @ R.T + eye)
    return np.concatenate(clouds, axis=0).astype(np.float32)


def capsule_points(seed: int = 3, n: int = 64, extent: float = 2.56, side: float = 0.005) -> np.ndarray:
    """Surfaces of n random capsules (radius U[0.02,0.10], length U[0.1,0.5])
    sampled at side/2 spacing."""
    rng = np.random.default_rng(seed)
    step = side / 2
    out = []
    for _ in range(n):
        r = rng.uniform(0.02, 0.10)
        length = rng.uniform(0.1, 0.5)
        c = rng.uniform(0.3, extent - 0.3, size=3)
        a = rng.normal(size=3)
        a /= np.linalg.norm(a)
        p0, p1 = c - a * length / 2, c + a * length / 2
        tmp = np.array([1.0, 0.0, 0.0]) if abs(a[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
        e1 = np.cross(a, tmp)
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(a, e1)
        n_ax = max(2, int(math.ceil(length / step)) + 1)
        n_ang = max(8, int(math.ceil(2 * math.pi * r / step)))
        s = np.linspace(0.0, 1.0, n_ax)[:, None, None]
        ang = np.linspace(0.0, 2 * math.pi, n_ang, endpoint=False)[None, :, None]
        ring = np.cos(ang) * e1 + np.sin(ang) * e2
        cyl = p0 + s * (p1 - p0) + r * ring
        out.append(cyl.reshape(-1, 3))
        n_sph = max(16, int(math.ceil(4 * math.pi * r * r / (step * step))))
        i = np.arange(n_sph) + 0.5
        phi = np.arccos(1 - 2 * i / n_sph)
        th = math.pi * (1 + 5 ** 0.5) * i
        sph = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], axis=1)
        along = sph @ a
        out.append(p1 + r * sph[along >= 0])
        out.append(p0 + r * sph[along < 0])
    return np.concatenate(out, axis=0).astype(np.float32)


# ---------------------------------------------------------------------------
# C3 / C4: arm, configurations, lists, trajectories
# ---------------------------------------------------------------------------

def arm_spec(n_joints: int = 7, spheres_per_link: int = 8) -> dict:
    """Synthetic 7-DOF DH arm (seed 4) with 8 spheres per link (seed 6)."""
    rng = np.random.default_rng(4)
    a = rng.uniform(0.1, 0.4, size=n_joints)
    d = rng.uniform(0.1, 0.4, size=n_joints)
    alpha = rng.choice(np.array([math.pi / 2, -math.pi / 2, 0.0]), size=n_joints)
    base = np.eye(4)
    base[:3, 3] = [1.28, 1.28, 0.1]
    srng = np.random.default_rng(6)
    n_s = n_joints * spheres_per_link
    return {
        "n_joints": n_joints,
        "base": base.reshape(-1).tolist(),
        "theta": [0.0] * n_joints,
        "d": d.tolist(),
        "a": a.tolist(),
        "alpha": alpha.tolist(),
        "link": [s // spheres_per_link for s in range(n_s)],
        "t": [((s % spheres_per_link) + 0.5) / spheres_per_link for s in range(n_s)],
        "r": srng.uniform(0.03, 0.08, size=n_s).tolist(),
    }


def c3_scene() -> MapScene:
    return MapScene((256, 256, 256), 0.01, box_scene(0, np.array([2.56, 2.56, 2.56])))


def c3_configs(n: int = 4096, n_joints: int = 7) -> np.ndarray:
    return np.random.default_rng(5).uniform(-math.pi, math.pi, size=(n, n_joints)).astype(np.float32)


def list_lengths(n_lists: int = 4096, lo: int = 2000, hi: int = 200_000) -> np.ndarray:
    rng = np.random.default_rng(7)
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_lists)).round().astype(np.int64)


def c3_lists_host(lengths: np.ndarray, n_vox: int, seed: int = 7):
    """Sorted unique uniform voxel ids per list (CSR), numpy; for small cases."""
    rng = np.random.default_rng(seed + 1000)
    ids, offs = [], [0]
    for L in lengths:
        v = np.unique(rng.integers(0, n_vox, size=int(L), dtype=np.int64)).astype(np.uint32)
        ids.append(v)
        offs.append(offs[-1] + v.shape[0])
    return np.concatenate(ids), np.asarray(offs, dtype=np.uint64)


def c3_lists_device(lengths: np.ndarray, n_vox: int, seed: int = 7, device: str = "cuda"):
    """Same shape of data generated on the device (torch Philox, seeded):
    per list uniform ids, sorted, duplicates dropped.  Returns (ids int32,
    offsets int64) CUDA tensors."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    L = torch.as_tensor(lengths, dtype=torch.int64, device=device)
    total = int(L.sum().item())
    owner = torch.repeat_interleave(torch.arange(L.shape[0], device=device), L)
    raw = torch.randint(0, n_vox, (total,), generator=g, device=device, dtype=torch.int64)
    key = torch.sort(owner * (1 << 32) + raw).values
    keep = torch.ones_like(key, dtype=torch.bool)
    keep[1:] = key[1:] != key[:-1]
    key = key[keep]
    owner = key >> 32
    ids = (key & 0xFFFFFFFF).to(torch.int32)
    counts = torch.bincount(owner, minlength=L.shape[0])
    offsets = torch.zeros(L.shape[0] + 1, dtype=torch.int64, device=device)
    offsets[1:] = torch.cumsum(counts, 0)
    return ids, offsets


def c4_points(n: int = 1_000_000, dims=(256, 256, 256), side: float = 0.01) -> np.ndarray:
    rng = np.random.default_rng(8)
    lo = 0.5 * side
    hi = (np.asarray(dims) - 0.5) * side
    return (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)


def c4_trajectories(n_traj: int = 512, n_wp: int = 64, n_joints: int = 7) -> np.ndarray:
    rng = np.random.default_rng(9)
    q0 = rng.uniform(-math.pi, math.pi, size=(n_traj, 1, n_joints))
    q1 = rng.uniform(-math.pi, math.pi, size=(n_traj, 1, n_joints))
    t = np.linspace(0.0, 1.0, n_wp)[None, :, None]
    return (q0 + (q1 - q0) * t).astype(np.float32)


# ---------------------------------------------------------------------------
# C5: many uneven maps
# ---------------------------------------------------------------------------

def c5_maps(n_maps: int = 64, lo: int = 64, hi: int = 384, side: float = 0.01):
    rng = np.random.default_rng(10)
    dims = np.exp(rng.uniform(math.log(lo), math.log(hi), size=(n_maps, 3))).round().astype(np.int64)
    npts = np.exp(rng.uniform(math.log(10_000), math.log(1_000_000), size=n_maps)).round().astype(np.int64)
    scenes = []
    for i in range(n_maps):
        extent = dims[i] * side
        scenes.append(MapScene(tuple(int(v) for v in dims[i]), side,
                               box_scene(100 + i, extent, n_points=int(npts[i]))))
    return scenes
