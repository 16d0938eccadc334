"""Host AMG setup (emg_amg.cpp): builds tests/amg_check.cpp against the
library's AMG source and runs it.  It checks, on a grid Laplacian with two
value parts, scalar and with three strongly coupled functions per vertex:
R = P^T, at most pmax entries per row of P, one identity row per coarse
unknown, Galerkin operators equal to R (A P) from two sparse products (1e-13)
and symmetric, and no interpolation across functions (the unknown approach of
systems AMG)."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_amg_hierarchy_invariants(tmp_path):
    cxx = shutil.which("g++")
    cuda = "/usr/local/cuda"
    if cxx is None or not os.path.isdir(os.path.join(cuda, "include")):
        pytest.skip("needs g++ and the CUDA headers")
    exe = tmp_path / "amg_check"
    src = os.path.join(ROOT, "emfem_b200", "csrc")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fopenmp", "-I", os.path.join(cuda, "include"), "-I", src,
                    os.path.join(ROOT, "tests", "amg_check.cpp"), os.path.join(src, "emg_amg.cpp"), "-o", str(exe),
                    "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(cuda, "lib64")],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
