"""The clusterizer's candidate box (hpgl_b200/csrc/plan.cpp: candidate_box),
which lets the clusterizer search skip the covariance read of candidates
that cannot pass its C(0)/100 test: checked against the model on every
integer offset around it, for seeded variograms of every type (built for the
host by tests/cpp/cand_box_check.cpp)."""

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_candidate_box_holds_every_passing_offset(tmp_path):
    out = str(tmp_path / "cand_box_check.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-pthread", "-o", out,
                    "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "cpp", "cand_box_check.cpp"),
                    os.path.join(ROOT, "hpgl_b200", "csrc", "plan.cpp")], check=True, capture_output=True)
    assert C.CDLL(out).cbc_run(7, 60) == 0
