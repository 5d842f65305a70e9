"""The host task pool (hpgl_b200/csrc/task_pool.cpp) that planning and the
staging copies run on: every index of a parallel loop exactly once for any
thread count, nested loops, exceptions reaching the caller after every
chunk finished (and the pool usable afterwards), concurrent callers, and
tasks that submit sub-tasks to their own group (built for the host by
tests/cpp/task_pool_check.cpp)."""

import ctypes as C
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def tpc(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("tpc") / "task_pool_check.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", out,
                    os.path.join(HERE, "cpp", "task_pool_check.cpp"),
                    os.path.join(ROOT, "hpgl_b200", "csrc", "task_pool.cpp")], check=True, capture_output=True)
    return C.CDLL(out)


@pytest.mark.parametrize("check", ["tpc_cover", "tpc_nested", "tpc_exception", "tpc_concurrent", "tpc_subtasks"])
def test_task_pool(tpc, check):
    assert getattr(tpc, check)() == 0
