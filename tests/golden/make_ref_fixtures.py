"""Generate golden fixtures from gpu-voxels' OWN kernels (oracle/_ref/libgvref.so,
built from the reference sources for sm_100a) -- needs a GPU.

    python tests/golden/make_ref_fixtures.py <out_dir> [lists]

Each fixture holds the seeded inputs' description and the reference's output
map after insertPointCloud + parallelBanding3D(1,1,1) (zlib-compressed), plus
the reference's squared distances and a BitVoxel collision count; the list
fixture holds the reference's per-list counts and marked list voxels of
LIST_CASE (`lists` makes only that one).  The CPU
test suite (tests/test_golden.py) checks the oracle against them without a GPU.
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "gpu-voxels_b200"), os.path.join(ROOT, "tests")]

import oracle  # noqa: E402
import refgeom  # noqa: E402
from golden_cases import CASES, LIST_CASE, list_inputs, points_for  # noqa: E402


def main(out_dir):
    R = oracle.ref_lib()
    assert R is not None and R.ref_available(), "reference kernels not built or no GPU"
    os.makedirs(out_dir, exist_ok=True)
    for name, spec in CASES.items():
        dims = tuple(spec["dims"])
        side = spec["side"]
        pts = points_for(spec)
        ins = oracle.dvm_empty(dims)
        flag = ctypes.c_int(0)
        rc = R.ref_dvm_insert(ins, np.asarray(dims, np.uint32), np.float32(side), np.ascontiguousarray(pts, np.float32),
                              pts.shape[0], ctypes.byref(flag))
        assert rc == 0
        edt = ins.copy()
        assert R.ref_pba(edt, np.asarray(dims, np.uint32), 1, 1, 1) == 0
        sq = oracle.sqdist_map(edt, dims)
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), dims=np.asarray(dims), side=np.float32(side),
                            inserted=ins, edt=edt, outside=np.int32(flag.value), sqdist_sum=np.int64(sq.astype(np.int64).sum()))
        print(name, dims, "outside", flag.value, "occupied", int((ins != oracle.DV_UNINIT).sum()))
    # BitVoxel collision known answer with the reference's kernel
    dims = (64, 64, 64)
    rng = np.random.default_rng(77)
    pa = (rng.random((30000, 3)) * 64).astype(np.float32)
    pb = (rng.random((30000, 3)) * 64).astype(np.float32)
    a, b = oracle.bvm_empty(dims), oracle.bvm_empty(dims)
    oracle.bvm_insert(a, dims, 1.0, pa, 1)
    oracle.bvm_insert(b, dims, 1.0, pb, 33)
    cnt = ctypes.c_uint64(0)
    a_ref = a.copy()
    assert R.ref_bvm_collide(a_ref, b, a.shape[0] // 32, ctypes.byref(cnt)) == 0
    np.savez_compressed(os.path.join(out_dir, "ref_bvm_collide.npz"), count=np.uint64(cnt.value), marked=a_ref)
    print("bvm collide", cnt.value)
    make_list_fixture(R, out_dir)


def make_list_fixture(R, out_dir):
    """Per-list counts and the marked list voxels of the reference's list-vs-map
    kernel, for every offset of LIST_CASE."""
    bmap, ids, vox, offs = list_inputs(LIST_CASE)
    dims = np.asarray(LIST_CASE["dims"], np.uint32)
    counts, marked = [], []
    for off in LIST_CASE["offsets"]:
        c = np.zeros(offs.shape[0] - 1, dtype=np.uint64)
        v = vox.copy()
        assert R.ref_lists_collide_map(ids, v, offs, c.shape[0], bmap, dims, np.asarray(off, np.int32), c) == 0
        counts.append(c)
        marked.append(v)
        print("list collide", off, c.tolist())
    np.savez_compressed(os.path.join(out_dir, "ref_list_collide.npz"), offsets=np.asarray(LIST_CASE["offsets"]),
                        counts=np.stack(counts), marked=np.stack(marked))


if __name__ == "__main__":
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden")
    if len(sys.argv) > 2 and sys.argv[2] == "lists":
        R = oracle.ref_lib()
        assert R is not None and R.ref_available(), "reference kernels not built or no GPU"
        os.makedirs(out, exist_ok=True)
        make_list_fixture(R, out)
    else:
        main(out)
