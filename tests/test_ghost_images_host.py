"""The ghost-entry writers of the projection update, run on the CPU.

``channel3d_parallel_b200/csrc/ghost_images.cuh`` (used by the time step's
projection kernel in place of a boundary-condition pass) is compiled with g++
against a host stand-in for the CUDA names it uses; filling every interior
point of u-, v- and w-shaped fields through it must reproduce the boundary
conditions entry for entry (periodic images, odd y reflections, zero v walls).
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_ghost_images_match_boundary_conditions(tmp_path):
    exe = str(tmp_path / "ghost_images_check")
    src = os.path.join(HERE, "host_kernels", "ghost_images_check.cpp")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(HERE, "host_kernels"), src, "-o", exe],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("0 mismatches") == 15
