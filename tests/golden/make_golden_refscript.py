"""Golden fixtures for the reference's own kriging test script
(python_pkg/misc/test/test.py:27-120 of the reference checkout) and its
test data (python_pkg/misc/test/test_data/: NEW_TEST_PROP.INC, a 55x52x1
continuous property with undefined value -99; NEW_TEST_PROP_01.INC, the
same cells as indicators 0/1; mp_0_8_52_55_1.inc, the locally varying
mean).

The inputs are read with the reference's own INC reader and every case is
run through the reference's own C ABI, both compiled from its sources by
oracle/build_ref.sh (oracle/_ref/libhpgl_ref.so).  The dump driver
(oracle/ref_dump.cpp) adds per-node neighbour lists, weights, variances and
statuses for a seeded sample of kriged nodes.

    python tests/golden/make_golden_refscript.py   # needs the reference checkout

The checkout is found by oracle.reference_src() ($HPGL_REFERENCE_SRC).
Writes tests/golden/refscript/<case>.npz, inputs included: the test data
itself is not needed to run the tests.

The script's parameters, in the geo_bsd API of the reference's current
Python layer (covariance types: spherical 0, exponential 1):

* ok:  exponential, ranges (10,10,10), sill 1, radii (20,20,20), 12 neighbours
* sk:  the same, mean 0.487 (and, as geo.simple_kriging(mean=None) gives it,
       the mean computed from the informed cells)
* lvm: the same variogram with the mean cube mp_0_8_52_55_1.inc
* median_ik: spherical, ranges (10,10,10), sill 0.4, radii (10,10,10),
       12 neighbours, marginal probabilities (0.5, 0.5) -- also what
       indicator_kriging with the script's two-category ik_data runs
* ik2: the script's ik_data through hpgl_indicator_kriging itself (full
       indicator kriging of both categories)
* ik4: the script's multi_ik_data (four spherical variograms with
       differing ranges, sills 0.25, radii (20,20,20), marginals 0.24,
       0.235, 0.34, 0.18) over the same codes, read with four indicator
       values.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hpgl_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden.make_golden import job_arrays  # noqa: E402

OUT = os.path.join(HERE, "refscript")
SHAPE = (55, 52, 1)
SIZE = SHAPE[0] * SHAPE[1] * SHAPE[2]


def _data_dir():
    return os.path.join(O.reference_src(), "python_pkg", "misc", "test", "test_data")


def _exp(**kw):
    return W.cov_params(1, (10, 10, 10), sill=1.0, radii=(20, 20, 20), max_neighbours=12, **kw)


def _sph04(marginal=0.0):
    return W.cov_params(0, (10, 10, 10), sill=0.4, radii=(10, 10, 10), max_neighbours=12, marginal_prob=marginal)


MULTI_IK = [((4, 4, 4), 0.24), ((6, 6, 6), 0.235), ((2, 2, 2), 0.34), ((10, 10, 10), 0.18)]


def cases():
    d = _data_dir()
    values, mask = O.ref_read_inc(os.path.join(d, "NEW_TEST_PROP.INC"), SIZE, -99.0)
    codes, cmask = O.ref_read_inc(os.path.join(d, "NEW_TEST_PROP_01.INC"), SIZE, -99, is_byte=True, values=(0, 1))
    mean, _ = O.ref_read_inc(os.path.join(d, "mp_0_8_52_55_1.inc"), SIZE, -99.0)
    cont = dict(shape=SHAPE, values=values, mask=mask)
    ind = dict(shape=SHAPE, codes=codes, mask=cmask)
    yield "ok", dict(cont, params=[_exp()]), "ok", {}
    yield "sk_mean0487", dict(cont, params=[_exp()], sk_mean=0.487), "sk", {}
    yield "sk_automatic_mean", dict(cont, params=[_exp()], sk_mean=0.0), "sk", {"sk_auto_mean": True}
    yield "lvm", dict(cont, params=[_exp()], mean=mean), "lvm", {}
    yield "median_ik", dict(ind, params=[_sph04()], median_marginal1=0.5), "median_ik", {}
    yield "ik2", dict(ind, params=[_sph04(0.5), _sph04(0.5)]), "ik", {}
    multi = [W.cov_params(0, r, sill=0.25, radii=(20, 20, 20), max_neighbours=12, marginal_prob=m) for r, m in MULTI_IK]
    yield "ik4", dict(ind, params=multi), "ik", {}


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libhpgl_ref.so not built (oracle/build_ref.sh)")
    os.makedirs(OUT, exist_ok=True)
    for name, job, kind, extra in cases():
        out, omask = O.ref_run(job, kind=kind, **extra)
        arrays = job_arrays(job, kind)
        arrays["sk_mean"] = np.float64(job.get("sk_mean", 0.0))
        arrays["sk_auto_mean"] = np.uint8(bool(extra.get("sk_auto_mean", False)))
        arrays["median_marginal1"] = np.float64(job.get("median_marginal1", 0.5))
        arrays["ref_out"] = out
        arrays["ref_mask"] = omask
        if not extra.get("sk_auto_mean"):
            cats = range(len(job["params"])) if kind == "ik" else [0]
            for k in cats:
                dump = O.ref_dump(job, kind=kind, category=k)
                kriged = np.nonzero(dump["status"] >= 0)[0]
                rng = np.random.default_rng(1000 + k)
                sample = np.sort(rng.choice(kriged, min(400, len(kriged)), replace=False)).astype(np.int32)
                sfx = "" if kind != "ik" else "_c%d" % k
                arrays["sample" + sfx] = sample
                arrays["ref_nb_count" + sfx] = dump["nb_count"][sample]
                arrays["ref_nb_index" + sfx] = dump["nb_index"].reshape(-1, dump["cap"])[sample]
                arrays["ref_weights" + sfx] = dump["weights"].reshape(-1, dump["cap"])[sample]
                arrays["ref_variance" + sfx] = dump["variance"][sample]
                arrays["ref_status" + sfx] = dump["status"][sample]
        path = os.path.join(OUT, name + ".npz")
        np.savez_compressed(path, **arrays)
        print("wrote", name, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
