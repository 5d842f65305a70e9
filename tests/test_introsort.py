"""The device restatement of the reference's std::sort (introsort.h) must
order equal keys exactly like libstdc++'s std::sort, which the reference
uses to rank clusterizer candidates (sugarbox_indexed_neighbour_lookup.h:99).
Compiles tests/cpp/introsort_check.cpp for the host and runs it on
tie-heavy inputs, including the heap-sort fallback."""

import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))


def test_introsort_matches_std_sort():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "introsort_check")
        subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe, os.path.join(HERE, "cpp", "introsort_check.cpp")],
                       check=True)
        r = subprocess.run([exe, "20000"], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        assert r.stdout.startswith("ok")
