"""Distance-field consumers on the GPU against the oracle, bit for bit:
extract_distances (free-space bytes, with and without a robot radius),
init_floodfill and extract_given_distances (distance band -> BitVoxelList)."""
import numpy as np
import pytest
import torch

import gvx
import oracle
from gpu_helpers import gpu_edt
import workloads

pytestmark = pytest.mark.gpu


def _scene(dims, side, seed, n=2000):
    return workloads.box_scene(seed, np.asarray(dims) * side, n_boxes=6, n_points=n).astype(np.float32)


@pytest.mark.parametrize("dims,r", [((64, 48, 40), 0), ((64, 48, 40), 5), ((33, 70, 17), 3), ((128, 128, 128), 0),
                                    ((20, 20, 20), 40)])
def test_extract_distances_and_floodfill(dims, r):
    pts = _scene(dims, 0.01, sum(dims))
    _, edt_g, dvm = gpu_edt(dims, 0.01, pts)
    want = oracle.extract_distances(edt_g, dims, r)
    got = dvm.extract_distances(r).cpu().numpy()
    assert np.array_equal(got, want)
    flood = dvm.init_floodfill(dvm.extract_distances(r), r).cpu().numpy()
    assert np.array_equal(flood, oracle.init_floodfill(want, r))


def test_extract_distances_of_an_empty_map_caps_at_127():
    dvm = gvx.DistanceVoxelMap((40, 30, 20), 0.01)
    assert (dvm.extract_distances(0) == 127).all()


@pytest.mark.parametrize("band", [(0, 0), (1, 3), (2, 127), (0, 127), (5, 2)])
def test_extract_given_distances(band):
    dims = (96, 80, 70)
    pts = _scene(dims, 0.01, 11, 3000)
    _, edt_g, dvm = gpu_edt(dims, 0.01, pts)
    ids_w, vox_w = oracle.extract_given_distances(edt_g, dims, *band)
    lst = gvx.BitVectorVoxelList(dims, 0.01)
    lst.insertPointCloud(torch.as_tensor(pts[:10]).cuda())  # earlier content is replaced
    n = gvx.extract_given_distances(dvm, band[0], band[1], lst)
    assert n == len(ids_w)
    assert np.array_equal(lst.ids().cpu().numpy().astype(np.uint32), ids_w)
    assert np.array_equal(lst.voxels().cpu().numpy().reshape(-1), vox_w)
