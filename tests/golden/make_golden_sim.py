"""Generates golden fixtures of sequential Gaussian and indicator simulation
from the reference's own sources compiled by oracle/build_ref.sh (with its
missing prime table generated by oracle/gen_primes.py and boost's mt11213b
from oracle/ref_shim): seeded inputs and the reference's simulated cubes.

    python tests/golden/make_golden_sim.py      # needs the reference build

Writes tests/golden/sim/<case>.npz."""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import oracle as O  # noqa: E402
import sis_cases as SC  # noqa: E402

OUT = os.path.join(HERE, "sim")


def calc_cdf(values, mask):
    v = np.asarray(values, np.float32)[np.asarray(mask) != 0]
    u, c = np.unique(v, return_counts=True)
    size = u.size - 1 if u.size > 1 else u.size
    return u[:size], np.cumsum(c[:size] / float(v.size)).astype(np.float32)


def sgs_cases():
    rng = np.random.default_rng(70)
    shape = (20, 18, 7)
    n = int(np.prod(shape))
    values = (rng.normal(size=n) * 2 + 1).astype(np.float32)
    mask = (rng.random(n) < 0.06).astype(np.uint8)
    p = dict(cov_type=1, ranges=(9.0, 6.0, 4.0), angles=(20.0, 0.0, 0.0), sill=1.0, nugget=0.1, radii=(10, 8, 5),
             max_neighbours=14)
    lvm = (0.3 * rng.normal(size=n)).astype(np.float32)
    sm = (rng.random(n) < 0.7).astype(np.uint8)
    cdf = calc_cdf(values, mask)
    yield "sgs_sk", dict(shape=shape, values=values, mask=mask, params=[p]), dict(seed=11)
    yield "sgs_ok_cdf", dict(shape=shape, values=values, mask=mask, params=[dict(p, cov_type=0)]), \
        dict(seed=12, ordinary=True, cdf=cdf)
    yield "sgs_lvm_mask_cdf", dict(shape=shape, values=values, mask=mask, params=[dict(p, max_neighbours=40)]), \
        dict(seed=13, lvm=lvm, sim_mask=sm, cdf=cdf)


def sis_cases():
    for K in (2, 3):
        c = SC.case(shape=(20, 16, 6), K=K, seed=80 + K)
        yield "sis_k%d" % K, c, SC.params(K), dict(seed=90 + K)
    c = SC.case(shape=(20, 16, 6), K=3, seed=85)
    ps = [dict(p, marginal_prob=0.0) for p in SC.params(3)]
    yield "sis_lvm_correlogram", c, ps, dict(seed=95, lvm=SC.means(c["shape"], 3, seed=86), correlogram=True)


def main():
    os.makedirs(OUT, exist_ok=True)
    for name, job, kw in sgs_cases():
        v, m = O.ref_sgs(job, **kw)
        extra = {k: kw[k] for k in ("lvm", "sim_mask") if k in kw}
        if "cdf" in kw:
            extra["cdf_values"], extra["cdf_probs"] = kw["cdf"]
        np.savez_compressed(os.path.join(OUT, name + ".npz"), kind=np.array("sgs"), shape=np.array(job["shape"]),
                            values=job["values"], mask=job["mask"], params=np.array(json.dumps(job["params"])),
                            seed=kw["seed"], ordinary=bool(kw.get("ordinary", False)), out_values=v, out_mask=m,
                            **extra)
        print(name)
    for name, c, ps, kw in sis_cases():
        codes, m = O.ref_sis(c["shape"], c["codes"], c["mask"], ps, **kw)
        extra = {}
        if "lvm" in kw:
            extra["lvm"] = np.array(kw["lvm"])
        np.savez_compressed(os.path.join(OUT, name + ".npz"), kind=np.array("sis"), shape=np.array(c["shape"]),
                            codes=c["codes"], mask=c["mask"], params=np.array(json.dumps(ps)), seed=kw["seed"],
                            correlogram=bool(kw.get("correlogram", False)), out_codes=codes, out_mask=m, **extra)
        print(name)


if __name__ == "__main__":
    main()
