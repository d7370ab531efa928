"""The shared-memory FFT engine of the CUDA library, run on the CPU.

``channel3d_parallel_b200/csrc/fft.cuh`` is compiled with g++ against a host
stand-in for the CUDA names it uses (one thread runs every butterfly); every
stage plan (radices 16, 12, 8, 6, 4, 3, 2) is checked against a long-double
DFT, with the digit-reversal maps and the inverse round trip.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_fft_engine_plans(tmp_path):
    exe = str(tmp_path / "fft_engine_check")
    src = os.path.join(HERE, "host_kernels", "fft_engine_check.cpp")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(HERE, "host_kernels"), src, "-o", exe],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "plan=16 12" in r.stdout      # N = 192 in two stages
