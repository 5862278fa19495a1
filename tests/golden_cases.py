"""Seeded input cases of the golden fixtures (tests/golden/ref_*.npz), inside
the reference's PBA domain (x == y, x % 64 == 0)."""
import numpy as np

import refgeom

CASES = {
    "random64": {"dims": (64, 64, 64), "side": 1.0, "kind": "uniform", "n": 400, "seed": 0},
    "lattice64x40": {"dims": (64, 64, 40), "side": 1.0, "kind": "lattice", "n": 100_000},
    "dense64": {"dims": (64, 64, 64), "side": 1.0, "kind": "uniform", "n": 60_000, "seed": 1},
    "symmetric": {"dims": (64, 64, 64), "side": 1.0, "kind": "fixed",
                  "pts": [[10.5, 32.5, 20.5], [53.5, 32.5, 20.5]]},
    "negative_and_outside": {"dims": (64, 64, 32), "side": 0.5, "kind": "uniform_wide", "n": 2000, "seed": 2},
    "boxes128x20": {"dims": (128, 128, 20), "side": 0.01, "kind": "boxes", "seed": 3},
}


def points_for(spec) -> np.ndarray:
    dims = np.asarray(spec["dims"], dtype=np.float64)
    side = spec["side"]
    kind = spec["kind"]
    if kind == "uniform":
        rng = np.random.default_rng(spec["seed"])
        return (rng.random((spec["n"], 3)) * dims * side).astype(np.float32)
    if kind == "uniform_wide":
        rng = np.random.default_rng(spec["seed"])
        return ((rng.random((spec["n"], 3)) * 1.4 - 0.2) * dims * side).astype(np.float32)
    if kind == "lattice":
        return refgeom.equidistant_points_fast(spec["n"], spec["dims"], side)
    if kind == "fixed":
        return np.asarray(spec["pts"], dtype=np.float32)
    if kind == "boxes":
        import workloads
        return workloads.box_scene(spec["seed"], dims * side, n_boxes=12, n_points=20_000)
    raise ValueError(kind)
