"""The CPU restatement of colocated simple cokriging (Markov models I and II,
oracle/hpgl_oracle.cpp) is pinned to the reference:

* against the committed golden fixtures (tests/golden/cokriging/*.npz,
  hpgl_simple_cokriging_mark1/2 of the reference's own sources compiled
  here -- tests/golden/make_golden_cokriging.py): estimate and mask of
  every node, bit for bit, including nodes without neighbours (the failure
  estimate) and ill-conditioned Gaussian systems;
* against the compiled reference itself on fresh seeded inputs, where the
  reference checkout was available to build it."""

import glob
import os

import numpy as np
import pytest

from hpgl_b200 import workloads as W
from oracle import oracle as O
from tests.golden.make_golden_cokriging import load

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "cokriging", "*.npz")))


def _same(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_cokriging_oracle_matches_golden(path):
    job, z = load(path)
    r = O.cokriging(job)
    assert _same(r["out"], z["ref_out"]), "estimates differ"
    assert np.array_equal(r["out_mask"], z["ref_mask"]), "masks differ"


@pytest.mark.skipif(not O.reference_available(), reason="compiled reference not present")
@pytest.mark.parametrize("mark", [1, 2])
def test_cokriging_oracle_matches_compiled_reference(mark):
    job = W.cokriging_job(shape=(30, 26, 9), mark=mark, seed=40 + mark, informed=0.03, max_neighbours=24)
    r = O.cokriging(job)
    out, mask = O.ref_cokriging(job)
    assert _same(r["out"], out)
    assert np.array_equal(r["out_mask"], mask)
