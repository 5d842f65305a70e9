"""The FP64 path divides by a diagonal entry through its correctly rounded
reciprocal plus one fused correction (Markstein); that must equal CUDA's
IEEE division bit for bit.  Compiles tests/cpp/division_check.cu and runs it
on the GPU over 2 x 10^8 random operand pairs."""

import os
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.gpu
def test_reciprocal_division_matches_ieee_division():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "division_check")
        subprocess.run(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                        "-std=c++17", "-o", exe, os.path.join(HERE, "cpp", "division_check.cu")], check=True)
        r = subprocess.run([exe, "100000000"], capture_output=True, text=True, timeout=300)
        print(r.stdout)
        assert r.returncode == 0, r.stdout + r.stderr
