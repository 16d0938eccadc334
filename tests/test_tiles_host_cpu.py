"""Row tiling for the tiled SpMM (emg_tiles.cpp): builds tests/tiles_check.cpp
against the library source and runs it (column lists ascending and within the
budget, local indices exact, the largest fitting tile height chosen,
impossible budgets refused)."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tile_rows(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("needs g++")
    exe = tmp_path / "tiles_check"
    src = os.path.join(ROOT, "emfem_b200", "csrc")
    subprocess.run([cxx, "-O2", "-std=c++17", "-fopenmp", "-I", src, os.path.join(ROOT, "tests", "tiles_check.cpp"),
                    os.path.join(src, "emg_tiles.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
