"""The maps' on-disk format is the reference's binary writeToDisk layout
(int32 MapType, float side, uint32 x y z, raw voxels): files written here
parse with that layout, files laid out that way read back, and reading
rejects another map type or other dims."""
import numpy as np
import pytest
import torch

import gvx
from gpu_helpers import gpu_edt, to_u32
import workloads

pytestmark = pytest.mark.gpu


def _header(path):
    raw = open(path, "rb").read()
    t = int(np.frombuffer(raw[:4], np.int32)[0])
    side = float(np.frombuffer(raw[4:8], np.float32)[0])
    dims = tuple(int(v) for v in np.frombuffer(raw[8:20], np.uint32))
    return t, side, dims, raw[20:]


def test_distance_map_round_trip_and_layout(tmp_path):
    dims = (40, 33, 21)
    pts = workloads.box_scene(5, np.asarray(dims) * 0.01, n_boxes=4, n_points=1500).astype(np.float32)
    _, edt, dvm = gpu_edt(dims, 0.01, pts)
    f = tmp_path / "dvm.gvm"
    dvm.writeToDisk(f)
    t, side, d, body = _header(f)
    assert t == 9 and d == dims and side == np.float32(0.01)
    assert np.array_equal(np.frombuffer(body, np.uint32), edt)
    back = gvx.DistanceVoxelMap(dims, 0.01)
    back.readFromDisk(f)
    assert np.array_equal(to_u32(back.data()), edt)
    with pytest.raises(gvx.GvxError):
        gvx.DistanceVoxelMap((40, 33, 22), 0.01).readFromDisk(f)
    with pytest.raises(gvx.GvxError):
        gvx.BitVectorVoxelMap(dims, 0.01).readFromDisk(f)
    other_side = gvx.DistanceVoxelMap(dims, 0.02)  # a different side only warns
    other_side.readFromDisk(f)
    assert np.array_equal(to_u32(other_side.data()), edt)


def test_bit_and_prob_maps_round_trip(tmp_path):
    dims = (24, 20, 16)
    rng = np.random.default_rng(0)
    pts = torch.as_tensor((rng.random((800, 3)) * np.asarray(dims) * 0.5).astype(np.float32)).cuda()
    b = gvx.BitVectorVoxelMap(dims, 0.5)
    b.insertPointCloud(pts, 7)
    b.insertPointCloud(pts[:100], 200)
    p = gvx.ProbVoxelMap(dims, 0.5)
    p.insertPointCloud(pts, 1)
    p.insertPointCloud(pts[:300], 0)
    for m, cls, code, view in [(b, gvx.BitVectorVoxelMap, 0, lambda x: x.voxels()),
                               (p, gvx.ProbVoxelMap, 4, lambda x: x.data())]:
        f = tmp_path / f"m{code}.gvm"
        m.writeToDisk(f)
        t, side, d, body = _header(f)
        assert t == code and d == dims and side == 0.5
        assert body == view(m).cpu().numpy().tobytes()
        r = cls(dims, 0.5)
        r.readFromDisk(f)
        assert torch.equal(view(r), view(m))


def test_reads_a_file_laid_out_by_hand(tmp_path):
    dims = (8, 6, 4)
    vox = np.full(np.prod(dims), 0x3FFFFFFF, np.uint32)
    vox[5] = 5 | (0 << 10) | (0 << 20)
    f = tmp_path / "hand.gvm"
    f.write_bytes(np.int32(9).tobytes() + np.float32(1.0).tobytes() + np.asarray(dims, np.uint32).tobytes() + vox.tobytes())
    m = gvx.DistanceVoxelMap(dims, 1.0)
    m.readFromDisk(f)
    assert np.array_equal(to_u32(m.data()), vox)
    f.write_bytes(f.read_bytes()[:-4])  # one voxel short
    with pytest.raises(gvx.GvxError):
        m.readFromDisk(f)
