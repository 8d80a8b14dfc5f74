"""The interior stage kernel's TMA halo boxes, checked on the CPU: a host
program (tests/native/tma_geometry.cu, compiled by nvcc against the kernels'
own header) sweeps grid sizes and CPML widths and checks every interior
tile's box start (16-byte aligned, non-negative), footprint and edge reads
before any of it runs on a GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "tma_geometry.cu")


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    return None


def test_interior_tma_boxes_are_aligned_and_in_bounds(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not found")
    exe = str(tmp_path / "tma_geometry")
    subprocess.check_call([nvcc, "-std=c++17", "-O1", "-gencode",
                           "arch=compute_100a,code=sm_100a", "-I",
                           os.path.join(ROOT, "include"), SRC, "-o", exe])
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok ") and int(r.stdout.split()[1]) > 1_000_000
