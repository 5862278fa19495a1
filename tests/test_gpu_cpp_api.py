"""The reference's own test scenarios through the gpu_voxels C++ API
(tests/cpp/test_gpu_voxels_api.cpp, built by the package Makefile)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "gpu-voxels_b200", "bin", "test_gpu_voxels_api")


def test_cpp_api_library_loads_without_gpu():
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "gpu-voxels_b200", "lib", "libgpu_voxels.so"))
    assert lib is not None
    assert os.path.exists(BIN)


@pytest.mark.gpu
def test_cpp_api_reference_scenarios():
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAIL" not in r.stdout
