"""torch autograd over the hand-written adjoint kernels.

The functions are libtorch C++ torch::autograd::Function subclasses
(torch_ext/gvx_torch.cpp) compiled in-tree into lib/torch_ext/ and linked
against lib/libgvx.so:

    d = trilinear_distance(points, dvm)            # [N,3] -> [N], d/dpoints by adjoint
    c = trajectory_cost(q, dvm, arm, margin=0.05)  # [B,T,J] -> [B], d/dq by adjoint
"""
from __future__ import annotations

import ctypes
import os

import torch

from ._abi import LIB_PATH, Arm

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_EXT_DIR = os.path.join(_PKG, "lib", "torch_ext")
_ROOT = os.path.dirname(_PKG)
_ext = None


def build(verbose: bool = False):
    """Compile (or reuse) the extension in lib/torch_ext/ and return the module."""
    global _ext
    if _ext is None:
        from torch.utils import cpp_extension

        os.makedirs(_EXT_DIR, exist_ok=True)
        lib_dir = os.path.dirname(LIB_PATH)
        _ext = cpp_extension.load(
            name="gvx_torch",
            sources=[os.path.join(_PKG, "torch_ext", "gvx_torch.cpp")],
            extra_include_paths=[os.path.join(_ROOT, "include")],
            extra_cflags=["-O2", "-std=c++17"],
            extra_ldflags=[f"-L{lib_dir}", "-lgvx", f"-Wl,-rpath,{lib_dir}"],
            build_directory=_EXT_DIR,
            with_cuda=True,
            verbose=verbose,
        )
    return _ext


def arm_blob(arm: Arm) -> torch.Tensor:
    """The gvx_arm struct as a CPU uint8 tensor (how the extension takes it)."""
    raw = ctypes.string_at(ctypes.addressof(arm), ctypes.sizeof(arm))
    return torch.frombuffer(bytearray(raw), dtype=torch.uint8).clone()


def trilinear_distance(points: torch.Tensor, dvm) -> torch.Tensor:
    return build().trilinear_distance(points, int(dvm.handle.value))


def trajectory_cost(q: torch.Tensor, dvm, arm: Arm, margin: float = 0.05) -> torch.Tensor:
    return build().trajectory_cost(q, int(dvm.handle.value), arm_blob(arm), float(margin))
