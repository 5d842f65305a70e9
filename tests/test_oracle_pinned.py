"""The CPU oracle (oracle/hpgl_oracle.cpp, the reference algorithm restated)
is itself pinned to the reference:

* against the committed golden fixtures (tests/golden/*.npz, produced by the
  reference's own sources compiled here — tests/golden/make_golden.py):
  estimates/categories, masks, and per-node neighbour lists, weights,
  variances and statuses, bit for bit;
* against the compiled reference itself (oracle/_ref, where the reference
  checkout was available) on fresh seeded inputs of every kind.
"""

import glob
import os

import numpy as np
import pytest

from hpgl_b200 import workloads as W
from oracle import oracle as O
from tests.golden.make_golden import load

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else (a.view(np.uint64) if a.dtype == np.float64 else a)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(path):
    job, kind, z = load(path)
    r = O.run(job, kind=kind)
    assert np.array_equal(_bits(r["out"]), _bits(z["ref_out"])), "outputs differ"
    assert np.array_equal(r["out_mask"], z["ref_mask"]), "masks differ"
    K = len(job["params"]) if kind == "ik" else 1
    slots = z["sample"].astype(np.int64) * K
    cap = r["cap"]
    assert np.array_equal(r["status"][slots], z["ref_status"].astype(np.int8))
    assert np.array_equal(r["nb_count"][slots], z["ref_nb_count"])
    nbi = r["nb_index"].reshape(-1, cap)[slots]
    w = r["weights"].reshape(-1, cap)[slots]
    for i, c in enumerate(z["ref_nb_count"]):
        assert np.array_equal(nbi[i, :c], z["ref_nb_index"][i, :c])
        if z["ref_status"][i] == 0:
            assert np.array_equal(_bits(w[i, :c]), _bits(z["ref_weights"][i, :c]))
    ok = z["ref_status"] == 0
    assert np.array_equal(_bits(r["variance"][slots][ok]), _bits(z["ref_variance"][ok]))


FRESH = {
    "ok": lambda: W.ok_50x50x20(shape=(30, 26, 12), seed=101),
    "sk": lambda: W.sk_ok_256x256x64(shape=(40, 36, 16), seed=102),
    "sk_auto_mean": lambda: W.sk_ok_256x256x64(shape=(40, 36, 16), seed=103),
    "lvm": lambda: W.lvm_512x512x32(shape=(64, 64, 10), seed=104, blobs=20),
    "ik": lambda: W.ik_200x200x100(shape=(30, 30, 12), seed=105),
    "median_ik": lambda: W.ik_200x200x100(shape=(30, 30, 12), seed=106, categories=2),
}


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built here")
@pytest.mark.parametrize("case", list(FRESH))
def test_oracle_matches_reference_abi(case):
    job = FRESH[case]()
    kind = {"sk_auto_mean": "sk"}.get(case, case)
    auto = case == "sk_auto_mean"
    r = O.run(job, kind=kind, sk_auto_mean=auto, dumps=False)
    out, mask = O.ref_run(job, kind=kind, sk_auto_mean=auto)
    assert np.array_equal(_bits(r["out"]), _bits(out))
    assert np.array_equal(r["out_mask"], mask)


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built here")
@pytest.mark.parametrize("case", ["ok", "sk", "lvm"])
def test_oracle_dumps_match_reference(case):
    job = FRESH[case]()
    r = O.run(job, kind=case)
    d = O.ref_dump(job, kind=case)
    kr = d["status"] >= 0
    assert np.array_equal(r["status"][kr], d["status"][kr].astype(np.int8))
    assert np.array_equal(r["nb_count"][kr], d["nb_count"][kr])
    cap = d["cap"]
    a = r["nb_index"].reshape(-1, cap)[kr]
    b = d["nb_index"].reshape(-1, cap)[kr]
    valid = np.arange(cap)[None, :] < d["nb_count"][kr][:, None]
    assert np.array_equal(a[valid], b[valid])
    ok = d["status"] == 0
    assert np.array_equal(_bits(r["variance"][ok]), _bits(d["variance"][ok]))
    wa = r["weights"].reshape(-1, cap)[ok]
    wb = d["weights"].reshape(-1, cap)[ok]
    v2 = np.arange(cap)[None, :] < d["nb_count"][ok][:, None]
    assert np.array_equal(_bits(wa[v2]), _bits(wb[v2]))


def test_template_matches_reference():
    p = W.sk_ok_256x256x64(shape=(8, 8, 8))["params"][0]
    t = O.template(p)
    assert len(t) > 0
    if O.reference_available():
        assert np.array_equal(t, O.ref_template(p))
