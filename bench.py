#!/usr/bin/env python
"""Benchmark of the distance-field collision path on B200.

Headline (one JSON line on rank 0): exact-EDT throughput in Gvoxel/s on the
512^3 @ 5 mm depth-image scene (voxelise ~1.2M points + EDT per step), with
the EDT kernels' HBM roofline, an end-to-end number through the public API
with host buffers (double-buffered: the next step's host->device copy runs on
a copy stream during this step; the serial loop is reported beside it), the
CPU oracle as a reported baseline and, when built,
gpu-voxels' own kernels timed on the same GPU.  Secondary sections cover the
other configs (128^3 queries, 512^3 BitVoxelMap collision, batched lists,
sphere/trajectory queries with gradients, many uneven maps).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU (one process per GPU): the headline is weak scaling -- every rank
voxelises and transforms its own 512^3 map, no collective on the data path;
the `sharded` section splits the independent units of configs C5 (64 uneven
maps) and C3 (4096 lists) over the ranks by a cost-balanced partition and
gathers the results on rank 0 (strong scaling).  Times = max over ranks.
"""
from __future__ import annotations

import argparse
import atexit
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-voxels_b200"))

import numpy as np  # noqa: E402

C2_DIMS = (512, 512, 512)
C2_SIDE = 0.005
EDT_BYTES_PER_VOXEL = 24  # 3 sweeps x (4 B read + 4 B write)
WORKLOAD = "c2_depth_scene_512cubed_5mm: voxelise ~1.23M pts + exact EDT"
PASS_BYTES_PER_VOXEL = 8


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling around the timed regions.

    The sampler starts before the warm-up (nvidia-smi takes a few hundred ms
    to deliver its first line) and stamps every sample with the host clock;
    `window()` marks a timed region, and the summary uses the samples taken
    inside the marked regions (or, if a region was shorter than the sampling
    interval, the sample nearest to each region)."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []  # (host time, fields)
        self.windows = []
        self._proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                           "--format=csv,noheader,nounits", "-lms", "50"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            atexit.register(self.stop)  # never leave the sampler running
            t0 = time.time()
            while not self.samples and time.time() - t0 < 3.0:  # first line before the workload starts
                time.sleep(0.02)
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append((time.time(), parts))

    def window(self):
        """Context manager marking one timed region (host time, synchronised edges)."""
        sampler = self

        class _W:
            def __enter__(self):
                self.t0 = time.time()
                return self

            def __exit__(self, *a):
                sampler.windows.append((self.t0, time.time()))

        return _W()

    def stop(self):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
            self._proc = None

    def summary(self):
        picked = [p for t, p in self.samples if any(a <= t <= b for a, b in self.windows)]
        if not picked and self.samples and self.windows:
            picked = [min(self.samples, key=lambda sp: min(abs(sp[0] - (a + b) / 2) for a, b in self.windows))[1]]
        if not picked:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in picked if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in picked if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in picked for i in range(4) if s[4 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(picked), "timed_windows": len(self.windows)}


def _traffic_from_profiles():
    """DRAM bytes per voxel of the EDT kernels from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "edt_kernels_c2_512cubed.txt")
    try:
        vals = {}
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_voxel"):
                    k, v = line.split(":", 1)
                    vals[k.strip()] = float(v.split()[0])
        return vals
    except Exception:
        return {}


class Ranks:
    """The bench's multi-process plumbing: one process per GPU (torchrun env),
    replicas with no data-path collective -- only a barrier around the timed
    region and the max of the per-rank times.  backend "nccl" on GPUs,
    "gloo" for the CPU tests of this logic."""

    def __init__(self, backend: str = "nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            from datetime import timedelta
            # bounded: after the collective steps rank 0 alone runs the baselines and the
            # config sections (about a minute) while the other ranks wait in close()
            dist.init_process_group(backend, timeout=timedelta(seconds=900))
            self.dist = dist

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def gpu_local_cpus(torch):
    """CPUs on the current GPU's NUMA node (NVML's affinity set), or None."""
    try:
        import pynvml
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
        h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        words = pynvml.nvmlDeviceGetCpuAffinity(h, ((os.cpu_count() or 64) + 63) // 64)
        cpus = {w * 64 + b for w, m in enumerate(words) for b in range(64) if (int(m) >> b) & 1}
        return (cpus & os.sched_getaffinity(0)) or None
    except Exception:
        return None


def pinned_near_gpu(torch, tensors):
    """Pinned host copies of `tensors`, allocated while this thread runs on the
    GPU's NUMA node so the pages land there (host->device copies from the far
    node run at a fraction of the link rate); the thread's affinity is restored."""
    cpus, before = gpu_local_cpus(torch), os.sched_getaffinity(0)
    if cpus:
        os.sched_setaffinity(0, cpus)
    try:
        out = [t.pin_memory() for t in tensors]
    finally:
        os.sched_setaffinity(0, before)
    return out, ("gpu-local NUMA node" if cpus else "default")


def bench_config(world: int) -> dict:
    """The workload description both arms print (identical keys and values)."""
    return {"workload": WORKLOAD, "map_dims": list(C2_DIMS), "voxel_side_m": C2_SIDE,
            "map_bytes": int(np.prod(C2_DIMS)) * 4,
            "l2": (f"map ({int(np.prod(C2_DIMS)) * 4 >> 20} MiB) larger than L2 (126 MB); no flush needed"
                   if np.prod(C2_DIMS) * 4 > 126e6 else "map fits in L2 (profiling case only)"),
            "parallelism": f"replicas x{world}"}


def whole_job_rate(units_per_rank: float, world: int, ms: float, scale: float = 1e9) -> float:
    """Throughput of the whole job: the units every rank processed over the
    slowest rank's time (ms), in units of `scale` per second."""
    return units_per_rank * world / (ms / 1e3) / scale


# ---------------------------------------------------------------------------
# reference arm: the CPU restatement (gpu-voxels has no CPU path of its own)
# ---------------------------------------------------------------------------

def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import workloads

    pts = workloads.c2_points()
    base = oracle.dvm_empty(C2_DIMS)
    oracle.dvm_insert(base, C2_DIMS, C2_SIDE, pts)
    times = []
    budget_s = 120.0  # the run stays within a few minutes whatever --steps asks for
    for it in range(args.warmup + args.steps):
        m = oracle.dvm_empty(C2_DIMS)
        t0 = time.perf_counter()
        oracle.dvm_insert(m, C2_DIMS, C2_SIDE, pts)
        oracle.pba(m, C2_DIMS)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
            if len(times) >= 3 and sum(times) > budget_s:
                break
    total = sum(times)
    nvox = float(np.prod(C2_DIMS))
    value = nvox * len(times) / total / 1e9
    cores = oracle.num_threads()
    line = {
        "impl": "reference", "metric": "edt_gvoxel_per_s", "value": round(value, 4), "unit": "Gvoxel/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * total / len(times), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32 (fp32 bisector)",
        "data": "synthetic", "config": bench_config(args.gpus),
        "cpu_baseline": {"value": round(value, 4), "unit": "Gvoxel/s", "cores": cores, "kind": "port",
                         "sample": "each step: insert + full 512^3 EDT of the C2 scene on the host cores (OpenMP)"},
        "e2e": {"value": round(value, 4), "unit": "Gvoxel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "steps_timed": len(times),
        "note": "gpu-voxels has no CPU implementation of this path; the arm runs the C restatement of its "
                "algorithm (oracle/gvx_oracle.c) on all host threads; timing stops after 120 s of steps",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# secondary sections (rank 0, after the headline)
# ---------------------------------------------------------------------------

def _time(fn, reps, warm=2):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps  # ms


def section_c1(hbm_peak):
    import torch
    import gvx
    import workloads
    sc = workloads.c1_scene()
    dvm = gvx.DistanceVoxelMap(sc.dims, sc.side)
    pts = torch.as_tensor(sc.points).cuda()
    ids = torch.as_tensor(workloads.c1_queries().astype(np.int32)).cuda()
    out = torch.empty_like(ids)
    nvox = int(np.prod(sc.dims))

    def edt():
        dvm.clearMap()
        dvm.insertPointCloud(pts)
        dvm.parallelBanding3D()

    ms_edt = _time(edt, 20)
    ms_q = _time(lambda: dvm.getSquaredDistances(ids, out=out), 50)
    return {"workload": "128^3 @ 1 cm, 50k box-scene points, 100k squared-distance queries",
            "voxelise_edt_ms": round(ms_edt, 4), "edt_gvoxel_per_s": round(nvox / ms_edt / 1e6, 3),
            "queries_per_s": round(ids.numel() / ms_q * 1e3, 1), "query_ms": round(ms_q, 4)}


def section_c2_collide(hbm_peak, pts_host):
    import torch
    import gvx
    import workloads
    dims = C2_DIMS
    nvox = int(np.prod(dims))
    scene = gvx.BitVectorVoxelMap(dims, C2_SIDE)
    caps = gvx.BitVectorVoxelMap(dims, C2_SIDE)
    scene.insertPointCloud(torch.as_tensor(pts_host).cuda(), 1)
    caps.insertPointCloud(torch.as_tensor(workloads.capsule_points()).cuda(), 4)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ms = _time(lambda: scene.collideWithAsync(caps, (0, 0, 0), True, cnt), 10)
    achieved = 64.0 * nvox / (ms / 1e3) / 1e9
    count = int(cnt.item())
    del scene, caps
    torch.cuda.empty_cache()
    return {"workload": "BitVectorVoxelMap 512^3 (depth scene) collideWith 512^3 (64 capsules)",
            "ms": round(ms, 4), "count": count, "achieved_gbs": round(achieved, 1),
            "frac_of_hbm": round(achieved / hbm_peak, 4), "algorithmic_bytes": 64 * nvox,
            "note": "the reference cannot allocate a 512^3 BitVoxelMap (32-bit byte limit)"}


def section_c3(hbm_peak):
    import torch
    import gvx
    import workloads
    sc = workloads.c3_scene()
    dvm = gvx.DistanceVoxelMap(sc.dims, sc.side)
    dvm.insertPointCloud(torch.as_tensor(sc.points).cuda())
    dvm.parallelBanding3D()
    arm = gvx.make_arm(workloads.arm_spec())
    q = torch.as_tensor(workloads.c3_configs()).cuda()
    n_cfg = q.shape[0]
    ms_batched = _time(lambda: dvm.sphere_clearance(arm, q), 20)
    cfg_views = [q[i:i + 1] for i in range(n_cfg)]
    ms_loop = _time(lambda: [dvm.sphere_clearance(arm, v) for v in cfg_views], 2, warm=1)
    n_sph = arm.n_spheres
    res = {"workload": "256^3 @ 1 cm scene; 4096 configs x 56 spheres; 4096 lists of 2k..200k ids",
           "sphere_queries_per_s": round(n_cfg * n_sph / ms_batched * 1e3, 1),
           "clearance_batched_ms": round(ms_batched, 4), "clearance_per_config_loop_ms": round(ms_loop, 3),
           "clearance_speedup_vs_loop": round(ms_loop / ms_batched, 1)}
    # lists vs the scene BitVoxelMap
    bmap = gvx.BitVectorVoxelMap(sc.dims, sc.side)
    bmap.insertPointCloud(torch.as_tensor(sc.points).cuda(), 1)
    lengths = workloads.list_lengths()
    ids, offs = workloads.c3_lists_device(lengths, int(np.prod(sc.dims)))
    n_ids = ids.numel()
    vox = torch.zeros(n_ids, 32, dtype=torch.uint8, device="cuda")
    owner = torch.repeat_interleave(torch.arange(len(lengths), device="cuda"), offs[1:] - offs[:-1])
    meaning = 4 + owner % 200
    vox.scatter_(1, (meaning // 8).unsqueeze(1), (1 << (meaning % 8)).to(torch.uint8).unsqueeze(1))
    vox = vox.reshape(-1)
    counts = torch.empty(len(lengths), dtype=torch.int64, device="cuda")
    ms_lb = _time(lambda: gvx.lists_collide_map(ids, vox, offs, bmap, counts=counts), 5)
    offs_h = offs.cpu().numpy()
    one = torch.empty(1, dtype=torch.int64, device="cuda")
    lens = offs[1:] - offs[:-1]
    local_offs = torch.stack([torch.zeros_like(lens), lens], 1).contiguous()  # [n_lists, 2]

    def per_list():
        for k in range(len(lengths)):
            a, b = int(offs_h[k]), int(offs_h[k + 1])
            gvx.lists_collide_map(ids[a:b], vox[a * 32:b * 32], local_offs[k], bmap, counts=one)
            _ = int(one.item())  # the reference returns each count to the host

    ms_ll = _time(per_list, 1, warm=1)
    # The batched call reduces the map to one occupancy bit per voxel (one
    # streaming read, 32 B per voxel, plus the bits written) when the lists
    # hold at least half as many entries as the map has voxels; then every
    # entry's id is read (4 B) and its 32-byte voxel only where the map bit is
    # set (every list voxel here holds a meaning, so those entries are the
    # hits).  Otherwise it gathers a 32-byte map voxel per entry (68 B per id).
    map_n = int(np.prod(sc.dims))
    bits_path = 2 * n_ids >= map_n
    hits_total = int(counts.sum().item())
    alg_bytes = (4.0 * n_ids + 32.0 * map_n + 4.0 * ((map_n + 31) // 32) + 32.0 * hits_total if bits_path
                 else 68.0 * n_ids)
    ach = alg_bytes / (ms_lb / 1e3) / 1e9
    res.update({"list_ids": int(n_ids), "lists_batched_ms": round(ms_lb, 4),
                "list_ids_per_s": round(n_ids / ms_lb * 1e3, 1),
                "lists_path": ("map occupancy bits (4 B/id + 32 B/voxel + 32 B per entry on an occupied voxel)"
                               if bits_path else "map gather (68 B/id)"),
                "lists_algorithmic_bytes": int(alg_bytes), "lists_achieved_gbs": round(ach, 1),
                "lists_frac_of_hbm": round(ach / hbm_peak, 4),
                "lists_per_list_loop_ms": round(ms_ll, 2), "lists_speedup_vs_loop": round(ms_ll / ms_lb, 1),
                "list_hits_total": int(counts.sum().item())})
    return res


def section_c4(hbm_peak):
    import torch
    import gvx
    import workloads
    from gvx import autograd
    sc = workloads.c3_scene()
    dvm = gvx.DistanceVoxelMap(sc.dims, sc.side)
    dvm.insertPointCloud(torch.as_tensor(sc.points).cuda())
    dvm.parallelBanding3D()
    pts = torch.as_tensor(workloads.c4_points()).cuda()
    n = pts.shape[0]
    gout = torch.ones(n, device="cuda")

    def fwd_bwd():
        d = dvm.trilinear(pts, with_grad=False)
        return dvm.trilinear_backward(pts, gout)

    gvx.set_query_config(256, 16)
    ms_fb_default = _time(fwd_bwd, 20)
    qcfg = dvm.autotune_queries(pts, with_grad=False, force=True)
    ms_fb = _time(fwd_bwd, 20)
    # the same points in cell order (z, y, x of the lower corner; sorted outside the timing):
    # neighbouring threads then share corner voxels and cache lines
    cell = torch.floor(pts / sc.side - 0.5).clamp_(min=0).to(torch.int64)
    key = (cell[:, 2] * sc.dims[1] + cell[:, 1]) * sc.dims[0] + cell[:, 0]
    pts_sorted = pts[torch.argsort(key)].contiguous()

    def fwd_bwd_sorted():
        dvm.trilinear(pts_sorted, with_grad=False)
        return dvm.trilinear_backward(pts_sorted, gout)

    ms_fb_sorted = _time(fwd_bwd_sorted, 20)
    p = pts.clone().requires_grad_(True)

    def autograd_step():
        p.grad = None
        autograd.trilinear_distance(p, dvm).sum().backward()

    ms_ag = _time(autograd_step, 20)
    arm = gvx.make_arm(workloads.arm_spec())
    q = torch.as_tensor(workloads.c4_trajectories()).cuda()
    B, T = q.shape[0], q.shape[1]
    gc = torch.ones(B, device="cuda")

    def traj():
        dvm.traj_cost(arm, q, 0.05)
        dvm.traj_cost_backward(arm, q, 0.05, gc)

    ms_tr = _time(traj, 10)
    views = [q[i:i + 1] for i in range(B)]
    gcv = gc[:1]

    def traj_loop():
        for v in views:
            dvm.traj_cost(arm, v, 0.05)
            dvm.traj_cost_backward(arm, v, 0.05, gcv)

    ms_trl = _time(traj_loop, 1, warm=1)
    bytes_fb = 48 + 60
    errors = c4_errors(dvm, sc, pts, arm, workloads)
    return {"errors_vs_fp64": errors,
            "workload": "256^3 map; 1M points trilinear fwd+bwd; 512 x 64 waypoints x 56 spheres hinge cost + adjoint",
            "trilinear_fwd_bwd_ms": round(ms_fb, 4), "trilinear_queries_with_grad_per_s": round(n / ms_fb * 1e3, 1),
            "query_launch_shape": {"threads": qcfg["threads"], "blocks_per_sm": qcfg["blocks_per_sm"],
                                   "fwd_bwd_ms_at_256x16": round(ms_fb_default, 4)},
            "trilinear_achieved_gbs": round(bytes_fb * n / (ms_fb / 1e3) / 1e9, 1),
            "trilinear_fwd_bwd_ms_cell_sorted": round(ms_fb_sorted, 4),
            "autograd_step_ms": round(ms_ag, 4),
            "traj_fwd_bwd_ms": round(ms_tr, 4),
            "traj_sphere_evals_with_grad_per_s": round(B * T * arm.n_spheres / ms_tr * 1e3, 1),
            "traj_per_trajectory_loop_ms": round(ms_trl, 2), "traj_speedup_vs_loop": round(ms_trl / ms_tr, 1)}


def c4_errors(dvm, sc, pts, arm, workloads):
    """Accuracy of the C4 queries (checker leg, outside every timed region):
    FP32 results against the FP64 oracle restatements of the same functions.
    Distances in voxel units; spatial gradients d(distance)/d(position)
    (dimensionless, so also voxel per voxel); the trajectory adjoint relative
    to the summed moment arms it is multiplied with (gcost * sum |z_k x
    (c_s - o_k)|_1 over the active spheres), i.e. in the same units as the
    spatial gradient."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    edt = dvm.data().cpu().numpy().view(np.uint32).copy()
    sample = pts[::5]  # 200k of the 1M points
    d32, g32 = dvm.trilinear(sample)
    xyz = sample.cpu().numpy()
    d64, g64 = oracle.trilinear64(edt, sc.dims, sc.side, xyz)
    derr = np.abs(d32.cpu().numpy().astype(np.float64) - d64) / sc.side
    u = xyz.astype(np.float64) / np.float64(np.float32(sc.side)) - 0.5
    fr = u - np.floor(u)
    off_face = ~np.any((fr < 1e-6) | (fr > 1 - 1e-6), axis=1)  # the gradient jumps across cell faces
    gerr = np.abs(g32.cpu().numpy().astype(np.float64) - g64)[off_face]
    spec = workloads.arm_spec()
    q = workloads.c4_trajectories(16, 64)
    gcost = np.ones(q.shape[0], dtype=np.float32)
    cost32 = dvm.traj_cost(arm, torch.as_tensor(q).cuda(), 0.05).cpu().numpy().astype(np.float64)
    gq = dvm.traj_cost_backward(arm, torch.as_tensor(q).cuda(), 0.05,
                                torch.as_tensor(gcost).cuda()).cpu().numpy().astype(np.float64)
    cost64 = oracle.traj_cost64(edt, sc.dims, sc.side, spec, q, 0.05)
    g64q, scale, gap = oracle.traj_cost_grad64(edt, sc.dims, sc.side, spec, q, 0.05, gcost)
    ok = np.broadcast_to((gap > 1e-6)[..., None], g64q.shape) & (scale > 0)
    rel = np.abs(gq - g64q)[ok] / scale[ok]
    return {
        "trilinear_points": int(xyz.shape[0]),
        "trilinear_err_max_vox": float(derr.max()), "trilinear_err_rms_vox": float(np.sqrt((derr ** 2).mean())),
        "grad_err_max": float(gerr.max()), "grad_err_rms": float(np.sqrt((gerr ** 2).mean())),
        "traj_cost_err_max_m": float(np.abs(cost32 - cost64).max()),
        "traj_cost_err_rel_max": float((np.abs(cost32 - cost64) / np.maximum(np.abs(cost64), 1e-30)).max()),
        "traj_adjoint_err_per_moment_arm_max": float(rel.max()),
        "traj_adjoint_err_per_moment_arm_rms": float(np.sqrt((rel ** 2).mean())),
        "traj_trajectories": int(q.shape[0]),
    }


def section_c5(hbm_peak):
    """64 uneven maps: voxelise + EDT + 10k trilinear distance/gradient queries
    each, as (a) a per-map loop of the plain calls, (b) the batch API eagerly
    (one launch per stage over all maps), (c) the batch step replayed as one
    CUDA graph.  The batch results are checked bit-equal to the loop's."""
    import torch
    import gvx
    import workloads
    from gvx.batch import Batch
    scenes = workloads.c5_maps()
    maps = [gvx.DistanceVoxelMap(s.dims, s.side) for s in scenes]
    pts_list = [torch.as_tensor(s.points).cuda() for s in scenes]
    pts = torch.cat(pts_list)
    offs = torch.zeros(len(scenes) + 1, dtype=torch.int64)
    offs[1:] = torch.cumsum(torch.tensor([p.shape[0] for p in pts_list]), 0)
    offs = offs.cuda()
    rng = np.random.default_rng(11)
    q_list, qm_list = [], []
    for k, s in enumerate(scenes):
        q_list.append(((0.5 + rng.random((10_000, 3)) * (np.asarray(s.dims) - 1)) * s.side).astype(np.float32))
        qm_list.append(np.full(10_000, k, dtype=np.int32))
    q = torch.as_tensor(np.concatenate(q_list)).cuda()
    qm = torch.as_tensor(np.concatenate(qm_list)).cuda()
    q_views = [q[k * 10_000:(k + 1) * 10_000] for k in range(len(scenes))]
    nvox = sum(int(np.prod(s.dims)) for s in scenes)

    def loop():
        for k, m in enumerate(maps):
            m.clearMap()
            m.insertPointCloud(pts_list[k])
            m.parallelBanding3D()
            m.trilinear(q_views[k])

    ms_loop = _time(loop, 3, warm=1)
    torch.cuda.synchronize()
    want = [m.data().clone() for m in maps]
    want_q = [m.trilinear(q_views[k]) for k, m in enumerate(maps)]
    b = Batch(maps)

    def eager():
        b.clear()
        b.insert(pts, offs)
        b.edt()
        b.query(q, qm)

    b.clear()
    b.insert(pts, offs)
    tuned = b.autotune()  # sweep configuration for these maps (timed on saved copies)
    ms_eager = _time(eager, 5)
    dist, grad = b.capture(pts, offs, q, qm)
    ms_graph = _time(b.replay, 10)
    torch.cuda.synchronize()
    exact = all(torch.equal(m.data(), w) for m, w in zip(maps, want))
    exact_q = all(torch.equal(dist[k * 10_000:(k + 1) * 10_000], want_q[k][0]) and
                  torch.equal(grad[k * 10_000:(k + 1) * 10_000], want_q[k][1]) for k in range(len(maps)))
    dims = [s.dims for s in scenes]
    return {"workload": "64 maps, dims log-uniform in [64,384] per axis, 10k-1M box-scene points each; "
                        "voxelise + exact EDT + 10k trilinear distance+gradient queries per map",
            "total_voxels": nvox, "total_points": int(pts.shape[0]), "min_dims": list(min(dims, key=np.prod)),
            "max_dims": list(max(dims, key=np.prod)),
            "per_map_loop_ms": round(ms_loop, 3), "batch_eager_ms": round(ms_eager, 3),
            "batch_graph_ms": round(ms_graph, 3),
            "loop_gvoxel_per_s": round(nvox / ms_loop / 1e6, 3), "graph_gvoxel_per_s": round(nvox / ms_graph / 1e6, 3),
            "graph_speedup_vs_loop": round(ms_loop / ms_graph, 2), "autotuned": tuned,
            "bit_equal_to_loop": bool(exact and exact_q)}


def section_sharded(ranks, steps: int, warmup: int):
    """The independent units of the path split over the ranks (every rank
    runs this; strong scaling: the total work is fixed as N grows).
      c5: the 64 uneven maps, voxelise + EDT + 10k trilinear queries per map,
          maps partitioned by voxel count; one Batch per rank.
      c3: the 4096 swept-volume lists against the 256^3 scene map, lists
          partitioned by length; one batched launch per rank.
    Time = max over ranks of the device time of `steps` steps (barrier and
    synchronize on both sides); the results are gathered on rank 0 after the
    timed region and checked against a single-GPU run of all units there."""
    import torch
    import gvx
    import workloads
    from gvx import shard
    from gvx.batch import Batch
    dist = ranks.dist
    out = {"scaling": "strong", "ranks": ranks.world}

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ranks.barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        ranks.barrier()
        torch.cuda.synchronize()
        return ranks.max(a.elapsed_time(b)) / steps

    scenes = workloads.c5_maps()
    rng = np.random.default_rng(11)
    queries = [((0.5 + rng.random((10_000, 3)) * (np.asarray(s.dims) - 1)) * s.side).astype(np.float32) for s in scenes]
    sb = shard.ShardedBatch(scenes, queries, dist)
    ms = timed(sb.step)
    full = sb.gather()
    nvox = sum(int(np.prod(s.dims)) for s in scenes)
    c5 = {"ms": round(ms, 4), "gvoxel_per_s": round(nvox / (ms / 1e3) / 1e9, 3), "maps_on_rank0": len(sb.mine),
          "imbalance": round(shard.imbalance(sb.costs, sb.plan), 4)}
    if ranks.rank == 0:  # the gathered results equal one GPU running every map (no collective here)
        try:
            maps = [gvx.DistanceVoxelMap(s.dims, s.side) for s in scenes]
            b = Batch(maps)
            pts = torch.as_tensor(np.concatenate([s.points for s in scenes]).astype(np.float32)).cuda()
            offs = torch.as_tensor(np.concatenate([[0], np.cumsum([s.points.shape[0] for s in scenes])])
                                   .astype(np.int64)).cuda()
            b.voxelize_edt(pts, offs)
            qm = torch.as_tensor(np.concatenate([np.full(q.shape[0], k, np.int32) for k, q in enumerate(queries)])).cuda()
            d, g = b.query(torch.as_tensor(np.concatenate(queries)).cuda(), qm)
            c5["equal_to_single_gpu"] = bool(torch.equal(full, torch.cat([d[:, None], g], 1)))
            del maps, b
        except Exception as exc:
            c5["check_error"] = repr(exc)[:200]
    del sb
    torch.cuda.empty_cache()
    out["c5_maps"] = c5

    sc = workloads.c3_scene()
    bmap = gvx.BitVectorVoxelMap(sc.dims, sc.side)
    bmap.insertPointCloud(torch.as_tensor(sc.points).cuda(), 1)
    ids, offs = workloads.c3_lists_device(workloads.list_lengths(), int(np.prod(sc.dims)))
    owner = torch.repeat_interleave(torch.arange(offs.shape[0] - 1, device="cuda"), offs[1:] - offs[:-1])
    meaning = 4 + owner % 200
    vox = torch.zeros(ids.numel(), 32, dtype=torch.uint8, device="cuda")
    vox.scatter_(1, (meaning // 8).unsqueeze(1), (1 << (meaning % 8)).to(torch.uint8).unsqueeze(1))
    vox = vox.reshape(-1)
    sl = shard.ShardedLists(ids, vox, offs.cpu().numpy(), bmap, dist)
    ms = timed(sl.step)
    counts = sl.gather()
    c3 = {"ms": round(ms, 4), "list_ids_per_s": round(ids.numel() / (ms / 1e3), 1), "lists_on_rank0": len(sl.mine),
          "imbalance": round(shard.imbalance(sl.lengths, sl.plan), 4)}
    if ranks.rank == 0:
        try:
            c3["equal_to_single_gpu"] = bool(torch.equal(counts, gvx.lists_collide_map(ids, vox, offs, bmap)))
        except Exception as exc:
            c3["check_error"] = repr(exc)[:200]
    out["c3_lists"] = c3
    del sl, ids, vox, bmap
    torch.cuda.empty_cache()
    return out


def run_sections(args, hbm_peak, pts_host):
    import torch
    out = {}
    for name, fn in (("c1_128", lambda: section_c1(hbm_peak)),
                     ("c2_collide_512", lambda: section_c2_collide(hbm_peak, pts_host)),
                     ("c3_spheres_lists", lambda: section_c3(hbm_peak)),
                     ("c4_gradients", lambda: section_c4(hbm_peak)),
                     ("c5_uneven_batch", lambda: section_c5(hbm_peak))):
        if args.sections not in ("all", "") and name not in args.sections.split(","):
            continue
        try:
            out[name] = fn()
        except Exception as exc:  # a failing section is reported, not fatal
            out[name] = {"error": repr(exc)[:300]}
        torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sections", default="all", help="comma list of extra sections or 'none'")
    ap.add_argument("--map", default="c2", choices=["c2", "c2_352", "c3"],
                    help="headline map: c2 = 512^3 depth scene (default), c2_352 = the same scene on a 352^3 map "
                         "(7.3 mm voxels; profiling captures), c3 = 256^3 box scene")
    ap.add_argument("--profile-sweeps", action="store_true",
                    help="for ncu captures: insert the map, then launch the y sweep, the x sweep and the fused "
                         "y->x sweep once each (16-row staging) and exit")
    ap.add_argument("--no-baselines", action="store_true", help="skip the CPU and reference-kernel baselines")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import gvx
    import workloads

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = Ranks("nccl")
    world, rank = ranks.world, ranks.rank
    barrier, max_over_ranks = ranks.barrier, ranks.max

    stream = torch.cuda.current_stream()
    hbm_peak, peak_kind = _peaks()

    # ---- headline workload, resident in HBM ------------------------------
    global C2_DIMS, C2_SIDE
    if args.map == "c3":  # the 256^3 @ 1 cm box scene (used for small profiling captures)
        sc = workloads.c3_scene()
        C2_DIMS, C2_SIDE, pts_host = sc.dims, sc.side, sc.points
    elif args.map == "c2_352":  # the depth scene on a smaller map (profiling captures above L2 size)
        C2_DIMS, C2_SIDE, pts_host = (352, 352, 352), 2.56 / 352, workloads.c2_points()
    else:
        pts_host = workloads.c2_points()
    if args.profile_sweeps:
        dvm = gvx.DistanceVoxelMap(C2_DIMS, C2_SIDE)
        dvm.set_edt_config(16, 1)
        pts = torch.as_tensor(pts_host).cuda()
        for p in (1, 2, 3):  # edt_sweep<Y>, edt_sweep<X>, edt_sweep_yx
            dvm.clearMap()
            dvm.insertPointCloud(pts)
            dvm.edt_pass(0)
            dvm.edt_pass(p)
        torch.cuda.synchronize()
        print(json.dumps({"profile_sweeps": list(C2_DIMS)}))
        ranks.close()
        return
    pts = torch.as_tensor(pts_host).cuda()
    dvm = gvx.DistanceVoxelMap(C2_DIMS, C2_SIDE)
    nvox = int(np.prod(C2_DIMS))

    def step():  # voxelise + exact EDT: clearMap + insertPointCloud + parallelBanding3D in one call
        dvm.voxelize_edt(pts)

    def three_calls():  # the same step as the reference's three calls
        dvm.clearMap()
        dvm.insertPointCloud(pts)
        dvm.parallelBanding3D()

    dvm.clearMap()
    dvm.insertPointCloud(pts)
    edt_config = dvm.autotune()  # untimed: picks the sweep configuration for this map
    clocks = ClockSampler(local).start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with clocks.window():
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = whole_job_rate(nvox * args.steps, world, ms)
    for _ in range(args.warmup):
        three_calls()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        three_calls()
    ev1.record(stream)
    torch.cuda.synchronize()
    three_ms = max_over_ranks(ev0.elapsed_time(ev1)) / args.steps

    # ---- kernel times of the EDT as parallelBanding3D runs it: the z sweep
    # (edt_pass_z) and the fused y -> x sweep (edt_sweep_yx); the y and x
    # sweeps launched separately are timed as well, for reference ----------
    def stage_times(stages):
        acc = [0.0] * len(stages)
        reps = max(5, args.steps)
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(len(stages) + 1)] for _ in range(reps)]
        for r in range(reps):
            dvm.clearMap()
            dvm.insertPointCloud(pts)
            e = evs[r]
            e[0].record(stream)
            for i, p in enumerate(stages):
                dvm.edt_pass(p)
                e[i + 1].record(stream)
        torch.cuda.synchronize()
        for r in range(reps):
            for i in range(len(stages)):
                acc[i] += evs[r][i].elapsed_time(evs[r][i + 1]) / reps
        return acc

    z_ms, yx_ms = stage_times([0, 3])
    sep_ms = stage_times([0, 1, 2])
    edt_ms = z_ms + yx_ms
    yx_bytes = 2 * PASS_BYTES_PER_VOXEL * nvox  # y sweep + x sweep: read + write each
    achieved = yx_bytes / (yx_ms / 1e3) / 1e9
    traffic = _traffic_from_profiles()
    tkey = "dram_bytes_per_voxel_edt_sweep_yx"
    roofline = {
        "bound": "hbm", "kernel": "edt_sweep_yx (fused y and x sweeps)", "achieved": round(achieved, 1),
        "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
        "traffic": (round(traffic[tkey] * nvox) if tkey in traffic else None),
        "algorithmic_bytes_per_launch": yx_bytes, "kernel_ms": round(yx_ms, 4),
        "pass_z_ms": round(z_ms, 4),
        "separate_passes_ms": {"z": round(sep_ms[0], 4), "y": round(sep_ms[1], 4), "x": round(sep_ms[2], 4)},
        "edt_total": {"ms": round(edt_ms, 4), "achieved_gbs": round(EDT_BYTES_PER_VOXEL * nvox / (edt_ms / 1e3) / 1e9, 1),
                      "frac": round(EDT_BYTES_PER_VOXEL * nvox / (edt_ms / 1e3) / 1e9 / hbm_peak, 4),
                      "gvoxel_per_s": round(nvox / (edt_ms / 1e3) / 1e9, 3)},
    }

    # ---- end to end through the public API with host buffers -------------
    (pinned, q_host, out_host, out_host2), pinned_where = pinned_near_gpu(torch, [
        torch.as_tensor(pts_host),
        torch.as_tensor(np.random.default_rng(1).integers(0, nvox, 100_000).astype(np.int32)),
        torch.empty(100_000, dtype=torch.int32), torch.empty(100_000, dtype=torch.int32)])
    pts_dev = torch.empty_like(pts)
    q_dev = torch.empty(q_host.shape[0], dtype=torch.int32, device="cuda")
    out_dev = torch.empty(q_host.shape[0], dtype=torch.int32, device="cuda")

    def e2e_step():
        pts_dev.copy_(pinned, non_blocking=True)
        q_dev.copy_(q_host, non_blocking=True)
        dvm.voxelize_edt(pts_dev)
        dvm.getSquaredDistances(q_dev, out=out_dev)
        out_host.copy_(out_dev, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    ev1.record(stream)
    torch.cuda.synchronize()
    serial_ms = max_over_ranks(ev0.elapsed_time(ev1))
    serial_out = out_host.clone()

    # The same steps double-buffered: step i+1's inputs cross on a copy stream
    # while step i runs, and step i's result returns on a third stream while
    # step i+1 runs; every step's H2D and D2H stay inside the timed region.
    copy_stream, d2h_stream = torch.cuda.Stream(), torch.cuda.Stream()
    pts_buf = [pts_dev, torch.empty_like(pts)]
    q_buf = [q_dev, torch.empty_like(q_dev)]
    out_devs = [out_dev, torch.empty_like(out_dev)]
    outs = [out_host, out_host2]
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    freed = [torch.cuda.Event(), torch.cuda.Event()]
    drained = [torch.cuda.Event(), torch.cuda.Event()]

    def e2e_pipelined(k_steps, start=None):
        for i in range(k_steps):
            b = i % 2
            with torch.cuda.stream(copy_stream):
                if i == 0 and start is not None:
                    copy_stream.wait_event(start)
                if i >= 2:
                    copy_stream.wait_event(freed[b])
                pts_buf[b].copy_(pinned, non_blocking=True)
                q_buf[b].copy_(q_host, non_blocking=True)
                copied[b].record(copy_stream)
            stream.wait_event(copied[b])
            if i >= 2:
                stream.wait_event(drained[b])  # step i-2's result has left out_devs[b]
            dvm.voxelize_edt(pts_buf[b])
            dvm.getSquaredDistances(q_buf[b], out=out_devs[b])
            freed[b].record(stream)
            with torch.cuda.stream(d2h_stream):
                d2h_stream.wait_event(freed[b])
                outs[b].copy_(out_devs[b], non_blocking=True)
                drained[b].record(d2h_stream)
        stream.wait_stream(d2h_stream)  # the last results are home before the step ends

    e2e_pipelined(args.warmup)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    with clocks.window():
        ev0.record(stream)
        e2e_pipelined(args.steps, start=ev0)
        ev1.record(stream)
        torch.cuda.synchronize()
    clocks.stop()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1))
    if not torch.equal(outs[(args.steps - 1) % 2], serial_out):
        raise RuntimeError("double-buffered end-to-end steps returned other distances than the serial steps")
    e2e = {"value": round(whole_job_rate(nvox * args.steps, world, e2e_ms), 3), "unit": "Gvoxel/s",
           "h2d_bytes_per_step": int(pinned.numel() * 4 + q_host.numel() * 4),
           "d2h_bytes_per_step": int(out_host.numel() * 4),
           "ms_per_step": round(e2e_ms / args.steps, 4),
           "path": "pinned points + query ids H2D, voxelize_edt (clearMap + insertPointCloud + "
                   "parallelBanding3D in one call), getSquaredDistances (100k ids), result D2H; "
                   "double-buffered: step i+1's H2D on a copy stream and step i's D2H on another "
                   "during step i+1",
           "serial": {"value": round(whole_job_rate(nvox * args.steps, world, serial_ms), 3),
                      "ms_per_step": round(serial_ms / args.steps, 4)},
           "pinned_memory": pinned_where}

    line = {
        "metric": "edt_gvoxel_per_s", "value": round(value, 3), "unit": "Gvoxel/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32 (fp32 bisector)",
        "data": "synthetic",
        "config": bench_config(world),
        "call": "voxelize_edt (clearMap + insertPointCloud + parallelBanding3D in one)",
        "three_call_step_ms": round(three_ms, 4),
        "roofline": roofline, "e2e": e2e, "edt_config": edt_config,
        "gpu_launches": 3 * args.steps,  # occupancy insert, z sweep from bits, fused y->x sweep (+ 2 memsets)
        "clocks": clocks.summary(),
    }

    # ---- the independent units split over the ranks (all ranks) ----------
    if args.sections == "all" or "sharded" in args.sections.split(","):
        try:
            line["sharded"] = section_sharded(ranks, steps=max(3, min(args.steps, 20)), warmup=3)
        except Exception as exc:  # reported, not fatal; every rank takes the same steps
            line["sharded"] = {"error": repr(exc)[:300]}

    if rank == 0 and not args.no_baselines:
        # ---- gpu-voxels' own kernels on this GPU (oracle/_ref), same map ----
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import ctypes
            import oracle
            R = oracle.ref_lib()
            if R is not None:
                ins = oracle.dvm_empty(C2_DIMS)
                oracle.dvm_insert(ins, C2_DIMS, C2_SIDE, pts_host)
                ms_ref = ctypes.c_float(0)
                rc = R.ref_pba_time(ins, np.asarray(C2_DIMS, np.uint32), 5, ctypes.byref(ms_ref))
                if rc == 0:
                    line["reference_cuda"] = {
                        "what": "gpu-voxels' own PBA kernels (m=1,1,1) built for sm_100a, same B200, same map",
                        "edt_ms": round(ms_ref.value, 3), "gvoxel_per_s": round(nvox / (ms_ref.value / 1e3) / 1e9, 3),
                        "our_edt_speedup": round(ms_ref.value / edt_ms, 2)}
            # ---- CPU oracle baseline (bounded sample: one full EDT) ----------
            m = oracle.dvm_empty(C2_DIMS)
            t0 = time.perf_counter()
            oracle.dvm_insert(m, C2_DIMS, C2_SIDE, pts_host)
            oracle.pba(m, C2_DIMS)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": round(nvox / dt / 1e9, 4), "unit": "Gvoxel/s",
                                    "cores": oracle.num_threads(), "kind": "port",
                                    "sample": "one insert + full 512^3 EDT of the same scene (OpenMP C restatement)"}
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}

    if rank == 0:
        if args.sections != "none":
            del dvm
            torch.cuda.empty_cache()
            line["sections"] = run_sections(args, hbm_peak, pts_host)
        print(json.dumps(line), flush=True)

    ranks.close()


if __name__ == "__main__":
    main()
