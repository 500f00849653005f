"""CPU check (no GPU) of the spatial-patch tables of the shared-memory Jacobi kernel: compiles tests/cpp/patch_check.cpp
against the product's host topology code (bevy_xpbd_b200/csrc/mesh_prep.cpp) with g++ and runs it."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cuda_include():
    for p in ("/usr/local/cuda/include", os.path.join(os.path.dirname(shutil.which("nvcc") or ""), "..", "include")):
        if os.path.exists(os.path.join(p, "vector_types.h")):
            return p
    return None


def test_patch_tables_reproduce_neighbour_rows(tmp_path):
    inc = _cuda_include()
    if inc is None or shutil.which("g++") is None:
        pytest.skip("g++ or CUDA headers not available")
    exe = str(tmp_path / "patch_check")
    csrc = os.path.join(ROOT, "bevy_xpbd_b200", "csrc")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", csrc, "-I", inc,
                           os.path.join(ROOT, "tests", "cpp", "patch_check.cpp"), os.path.join(csrc, "mesh_prep.cpp"),
                           "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
