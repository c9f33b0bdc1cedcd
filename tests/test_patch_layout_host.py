"""The fused step's patch records checked on the host (no GPU): builds
tests/cpp/check_patch_layout.cc against akantu_b200/csrc/akb_patch_build.cu
with nvcc (host code only) and runs it. It checks, on tetrahedral,
hexahedral, triangular and segment meshes (structured, scrambled, a star of
elements around one node, several patch sizes, FP64 and FP32 slot
colourings, pieces of 1 to 8 contributions): every shared-memory index a
record yields stays inside its buffer, the contribution slots of a chunk
are a bijection, the two levels of piece sums give each node exactly the
sum of its contributions, node positions are distinct, every element is in
one patch, and the coloured scatter and sum instructions hit distinct
banks."""
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.timeout(600)
def test_patch_records_on_host():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "check_patch_layout")
        subprocess.run([nvcc, "-std=c++17", "-O2",
                        "-I", os.path.join(ROOT, "akantu_b200", "csrc"),
                        "-I", os.path.join(ROOT, "include"),
                        "-o", exe, os.path.join(ROOT, "tests", "cpp", "check_patch_layout.cc"),
                        os.path.join(ROOT, "akantu_b200", "csrc", "akb_patch_build.cu")],
                       check=True, capture_output=True, text=True)
        out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "fails 0" in out.stdout
