"""CPU: the oracle reproduces gpu-voxels' own kernel outputs bit for bit
(fixtures produced on a B200 by tests/golden/make_ref_fixtures.py)."""
import glob
import os

import numpy as np
import pytest

import oracle
from golden_cases import CASES, points_for

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(glob.glob(os.path.join(HERE, "ref_*.npz")))


def test_fixtures_present():
    assert any("ref_random64" in f for f in FIXTURES), "golden fixtures missing"


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_kernels(name):
    path = os.path.join(HERE, f"ref_{name}.npz")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    f = np.load(path)
    spec = CASES[name]
    dims = tuple(int(v) for v in f["dims"])
    pts = points_for(spec)
    m = oracle.dvm_empty(dims)
    outside = oracle.dvm_insert(m, dims, float(f["side"]), pts)
    assert np.array_equal(m, f["inserted"]), "voxelisation differs from the reference kernel"
    assert int(outside) == int(f["outside"])
    oracle.pba(m, dims)
    assert np.array_equal(m, f["edt"]), f"EDT differs at {int(np.count_nonzero(m != f['edt']))} voxels"
    lit = f["inserted"].copy()
    oracle.pba_reference_order(lit, dims)
    assert np.array_equal(lit, f["edt"])


def test_oracle_collision_matches_reference_kernel():
    path = os.path.join(HERE, "ref_bvm_collide.npz")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    f = np.load(path)
    dims = (64, 64, 64)
    rng = np.random.default_rng(77)
    pa = (rng.random((30000, 3)) * 64).astype(np.float32)
    pb = (rng.random((30000, 3)) * 64).astype(np.float32)
    a, b = oracle.bvm_empty(dims), oracle.bvm_empty(dims)
    oracle.bvm_insert(a, dims, 1.0, pa, 1)
    oracle.bvm_insert(b, dims, 1.0, pb, 33)
    assert oracle.bvm_collide(a, b) == int(f["count"])
    assert np.array_equal(a, f["marked"])


def test_oracle_list_collision_matches_reference_kernel():
    """The oracle's list-vs-map restatement against the reference's own
    kernelCollideWithVoxelMap: per-list counts and the collision marks left
    in the list voxels, at four map offsets (one list entry per id; ids beyond
    the map and free-only voxels included)."""
    from golden_cases import LIST_CASE, linear_offset, list_inputs

    path = os.path.join(HERE, "ref_list_collide.npz")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    f = np.load(path)
    bmap, ids, vox, offs = list_inputs(LIST_CASE)
    dims = LIST_CASE["dims"]
    assert [tuple(o) for o in f["offsets"]] == [tuple(o) for o in LIST_CASE["offsets"]]
    for k, off in enumerate(LIST_CASE["offsets"]):
        lin = linear_offset(dims, off)
        v = vox.copy()
        got = []
        for l in range(offs.shape[0] - 1):
            a, b = int(offs[l]), int(offs[l + 1])
            seg = v[a * 32:b * 32].copy()
            got.append(oracle.list_collide_map(ids[a:b], seg, bmap, lin, True))
            v[a * 32:b * 32] = seg
        assert got == [int(c) for c in f["counts"][k]], off
        assert np.array_equal(v, f["marked"][k]), off
    assert int(f["counts"].sum()) > 0
