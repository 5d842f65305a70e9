"""Node coordinates on the device divide by the grid extents with a
multiply-high (FastDiv in hpgl_b200/csrc/kernels.cuh, Granlund-Montgomery).
Compiles tests/cpp/fastdiv_check.cpp for the host and compares it with
integer division on every divisor up to 4096, the grid extents up to 2^16
and their edge numerators."""

import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))


def test_fastdiv_matches_integer_division():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "fastdiv_check")
        subprocess.run(["g++", "-O2", "-std=c++17", "-I/usr/local/cuda/include", "-o", exe,
                        os.path.join(HERE, "cpp", "fastdiv_check.cpp")], check=True)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        assert r.stdout.startswith("ok")
