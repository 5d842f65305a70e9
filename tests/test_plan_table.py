"""The plan's covariance table (hpgl_b200/csrc/plan.cpp), which reuses the
search template's box of C(-v) when the table covers the same box, equals
the table evaluated from the model bit for bit, and its search template,
sorted with sub-ranges on the planning threads, equals the template rebuilt
on one thread (built for the host by tests/cpp/plan_table_check.cpp)."""

import ctypes as C
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_table_from_template_box_is_exact(tmp_path):
    out = str(tmp_path / "plan_table_check.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-pthread", "-o", out,
                    "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "cpp", "plan_table_check.cpp"),
                    os.path.join(ROOT, "hpgl_b200", "csrc", "plan.cpp"),
                    os.path.join(ROOT, "hpgl_b200", "csrc", "task_pool.cpp")], check=True, capture_output=True)
    assert C.CDLL(out).ptc_run(11, 40) == 0


@pytest.mark.parametrize("threads", [1, 3, 8])
def test_template_order_independent_of_threads(tmp_path, threads):
    """The template sorted with sub-ranges on pool threads equals the one
    rebuilt on one thread with the sequential reference sort."""
    out = str(tmp_path / "plan_table_check.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-pthread", "-o", out,
                    "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "cpp", "plan_table_check.cpp"),
                    os.path.join(ROOT, "hpgl_b200", "csrc", "plan.cpp"),
                    os.path.join(ROOT, "hpgl_b200", "csrc", "task_pool.cpp")], check=True, capture_output=True)
    assert C.CDLL(out).ptc_template(7 + threads, 6, threads) == 0
