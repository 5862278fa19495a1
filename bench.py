#!/usr/bin/env python
"""Benchmark of the distance-field collision path on B200.

Headline (one JSON line on rank 0): exact-EDT throughput in Gvoxel/s on the
512^3 @ 5 mm depth-image scene (voxelise ~1.2M points + EDT per step), with
the EDT kernels' HBM roofline, an end-to-end number through the public API
with host buffers, the CPU oracle as a reported baseline and, when built,
gpu-voxels' own kernels timed on the same GPU.  Secondary sections cover the
other configs (128^3 queries, 512^3 BitVoxelMap collision, batched lists,
sphere/trajectory queries with gradients, many uneven maps).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: every rank runs its own independent map (weak scaling, no
collective on the data path); time = max over ranks.
"""
from __future__ import annotations

import argparse
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
PASS_BYTES_PER_VOXEL = 8


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                           "--format=csv,noheader,nounits", "-lms", "100"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[4 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def _traffic_from_profiles():
    """DRAM bytes per voxel of the dominant EDT pass from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "edt_passes_512.txt")
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


# ---------------------------------------------------------------------------
# reference arm: the CPU restatement (gpu-voxels has no CPU path of its own)
# ---------------------------------------------------------------------------

def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from gvx import workloads

    pts = workloads.c2_points()
    base = oracle.dvm_empty(C2_DIMS)
    oracle.dvm_insert(base, C2_DIMS, C2_SIDE, pts)
    times = []
    for it in range(args.warmup + args.steps):
        m = oracle.dvm_empty(C2_DIMS)
        t0 = time.perf_counter()
        oracle.dvm_insert(m, C2_DIMS, C2_SIDE, pts)
        oracle.pba(m, C2_DIMS)
        dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
    total = sum(times)
    nvox = float(np.prod(C2_DIMS))
    value = nvox * len(times) / total / 1e9
    cores = oracle.num_threads()
    line = {
        "impl": "reference", "metric": "edt_gvoxel_per_s", "value": round(value, 4), "unit": "Gvoxel/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * total / len(times), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32 (fp32 bisector)",
        "data": "synthetic", "config": {"workload": "c2_depth_scene_512cubed_5mm: voxelise ~1.23M pts + exact EDT"},
        "cpu_baseline": {"value": round(value, 4), "unit": "Gvoxel/s", "cores": cores, "kind": "port",
                         "sample": "each step: insert + full 512^3 EDT of the C2 scene on the host cores (OpenMP)"},
        "e2e": {"value": round(value, 4), "unit": "Gvoxel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "gpu-voxels has no CPU implementation of this path; the arm runs the C restatement of its "
                "algorithm (oracle/gvx_oracle.c) on all host threads",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sections", default="all", help="comma list of extra sections or 'none'")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import gvx
    from gvx import workloads

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    stream = torch.cuda.current_stream()
    hbm_peak, peak_kind = _peaks()

    # ---- C2 workload, resident in HBM ------------------------------------
    pts_host = workloads.c2_points()
    pts = torch.as_tensor(pts_host).cuda()
    dvm = gvx.DistanceVoxelMap(C2_DIMS, C2_SIDE)
    nvox = int(np.prod(C2_DIMS))

    def step():
        dvm.clearMap()
        dvm.insertPointCloud(pts)
        dvm.parallelBanding3D()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = nvox * args.steps * world / (ms / 1e3) / 1e9

    # ---- per-pass kernel times (dominant kernel roofline) -----------------
    pass_ms = [0.0, 0.0, 0.0]
    reps = max(5, args.steps)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(reps)]
    for r in range(reps):
        dvm.clearMap()
        dvm.insertPointCloud(pts)
        e = evs[r]
        e[0].record(stream)
        for p in range(3):
            dvm.edt_pass(p)
            e[p + 1].record(stream)
    torch.cuda.synchronize()
    for r in range(reps):
        for p in range(3):
            pass_ms[p] += evs[r][p].elapsed_time(evs[r][p + 1]) / reps
    edt_ms = sum(pass_ms)
    dom = int(np.argmax(pass_ms))
    pass_names = ["edt_pass_z", "edt_pass_y", "edt_pass_x"]
    achieved = PASS_BYTES_PER_VOXEL * nvox / (pass_ms[dom] / 1e3) / 1e9
    traffic = _traffic_from_profiles()
    tkey = f"dram_bytes_per_voxel_{pass_names[dom]}"
    roofline = {
        "bound": "hbm", "kernel": pass_names[dom], "achieved": round(achieved, 1), "peak": hbm_peak,
        "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
        "traffic": (round(traffic[tkey] * nvox) if tkey in traffic else None),
        "algorithmic_bytes_per_launch": PASS_BYTES_PER_VOXEL * nvox,
        "per_pass_ms": [round(x, 4) for x in pass_ms],
        "edt_total": {"ms": round(edt_ms, 4), "achieved_gbs": round(EDT_BYTES_PER_VOXEL * nvox / (edt_ms / 1e3) / 1e9, 1),
                      "frac": round(EDT_BYTES_PER_VOXEL * nvox / (edt_ms / 1e3) / 1e9 / hbm_peak, 4),
                      "gvoxel_per_s": round(nvox / (edt_ms / 1e3) / 1e9, 3)},
    }

    # ---- end to end through the public API with host buffers -------------
    pinned = torch.as_tensor(pts_host).pin_memory()
    q_host = torch.as_tensor(np.random.default_rng(1).integers(0, nvox, 100_000).astype(np.int32)).pin_memory()
    out_host = torch.empty(q_host.shape[0], dtype=torch.int32).pin_memory()
    pts_dev = torch.empty_like(pts)
    q_dev = torch.empty(q_host.shape[0], dtype=torch.int32, device="cuda")
    out_dev = torch.empty(q_host.shape[0], dtype=torch.int32, device="cuda")

    def e2e_step():
        pts_dev.copy_(pinned, non_blocking=True)
        q_dev.copy_(q_host, non_blocking=True)
        dvm.clearMap()
        dvm.insertPointCloud(pts_dev)
        dvm.parallelBanding3D()
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
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1))
    e2e = {"value": round(nvox * args.steps * world / (e2e_ms / 1e3) / 1e9, 3), "unit": "Gvoxel/s",
           "h2d_bytes_per_step": int(pinned.numel() * 4 + q_host.numel() * 4),
           "d2h_bytes_per_step": int(out_host.numel() * 4),
           "ms_per_step": round(e2e_ms / args.steps, 4),
           "path": "pinned points + query ids H2D, clearMap, insertPointCloud, parallelBanding3D, "
                   "getSquaredDistances (100k ids), result D2H"}

    line = {
        "metric": "edt_gvoxel_per_s", "value": round(value, 3), "unit": "Gvoxel/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32 (fp32 bisector)",
        "data": "synthetic",
        "config": {"workload": "c2_depth_scene_512cubed_5mm: clearMap + insertPointCloud(~1.23M pts) + exact EDT",
                   "map_bytes": nvox * 4, "l2": "map (512 MiB) larger than L2; no flush needed",
                   "parallelism": f"replicas x{world}"},
        "roofline": roofline, "e2e": e2e,
        "gpu_launches": 5 * args.steps,
        "clocks": clocks.summary(),
    }

    if rank == 0:
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

        if args.sections != "none":
            try:
                import bench_sections
                line["sections"] = bench_sections.run_all(args, dvm, pts, hbm_peak)
            except Exception as exc:
                line["sections"] = {"error": repr(exc)[:300]}
        print(json.dumps(line), flush=True)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
