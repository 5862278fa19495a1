"""Shared helpers of the GPU parity tests (call the C ABI through gvx)."""
import numpy as np
import torch

import gvx
import oracle


def to_u32(t: torch.Tensor) -> np.ndarray:
    return t.detach().cpu().numpy().view(np.uint32).copy()


def gpu_edt(dims, side, pts, m=1):
    """insert + EDT on the GPU; returns (map after insert, map after EDT) as numpy uint32."""
    dvm = gvx.DistanceVoxelMap(dims, side)
    dvm.insertPointCloud(torch.as_tensor(np.asarray(pts, dtype=np.float32)))
    before = to_u32(dvm.data())
    dvm.parallelBanding3D(m, m, m)
    after = to_u32(dvm.data())
    return before, after, dvm


def oracle_edt(dims, side, pts):
    m = oracle.dvm_empty(dims)
    oracle.dvm_insert(m, dims, side, pts)
    ins = m.copy()
    oracle.pba(m, dims)
    return ins, m


def first_mismatch(a: np.ndarray, b: np.ndarray, dims):
    bad = np.nonzero(a != b)[0]
    if bad.size == 0:
        return None
    i = int(bad[0])
    X, Y = dims[0], dims[1]
    return dict(count=int(bad.size), id=i, pos=(i % X, (i // X) % Y, i // (X * Y)), got=hex(int(a[i])), want=hex(int(b[i])))
