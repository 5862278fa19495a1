"""gvx: B200-native distance-field collision engine with the gpu-voxels API.

The compute path is lib/libgvx.so (hand-written sm_100a CUDA behind the C ABI
in include/gvx.h).  This package is the Python face of that ABI: map handles
named after the reference classes, synthetic workload generators and the
torch autograd functions.
"""
from ._abi import GvxError, LIB_PATH, lib  # noqa: F401
from .maps import (  # noqa: F401
    BIT_VECTOR_LENGTH,
    BitVectorVoxelList,
    BitVectorVoxelMap,
    DistanceVoxelMap,
    ProbVoxelMap,
    eBVM_COLLISION,
    eBVM_FREE,
    eBVM_OCCUPIED,
    extract_given_distances,
    lists_collide_map,
    make_arm,
    set_query_config,
)

__all__ = [
    "GvxError",
    "LIB_PATH",
    "lib",
    "DistanceVoxelMap",
    "BitVectorVoxelMap",
    "BitVectorVoxelList",
    "ProbVoxelMap",
    "lists_collide_map",
    "extract_given_distances",
    "make_arm",
    "set_query_config",
    "BIT_VECTOR_LENGTH",
    "eBVM_FREE",
    "eBVM_OCCUPIED",
    "eBVM_COLLISION",
]
