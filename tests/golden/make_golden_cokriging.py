"""Generates the golden fixtures of colocated simple cokriging (Markov models
I and II) from the reference's own sources compiled by oracle/build_ref.sh:
for small seeded inputs, the reference's C-ABI outputs of
hpgl_simple_cokriging_mark1/2 (estimate and mask of every node), inputs
included.

    python tests/golden/make_golden_cokriging.py      # needs the reference checkout

Writes tests/golden/cokriging/<case>.npz."""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hpgl_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def _with(job, **p):
    job["params"] = [dict(job["params"][0], **p)]
    return job


CASES = {
    "cok1_spherical_n16_40x40x10": lambda: W.cokriging_job(shape=(40, 40, 10), mark=1, seed=21),
    "cok2_exponential2_n16_40x40x10": lambda: W.cokriging_job(shape=(40, 40, 10), mark=2, seed=22),
    # sparse primary, small search box: many nodes without neighbours (the
    # failure estimate m1 + s - m2), half the secondary missing
    "cok1_sparse_32x32x8": lambda: _with(W.cokriging_job(shape=(32, 32, 8), mark=1, seed=23, informed=0.004,
                                                         secondary_informed=0.5), radii=(4, 4, 2)),
    # Gaussian primary model, 48 neighbours: ill-conditioned eliminations
    "cok2_gaussian_n48_36x36x8": lambda: _with(W.cokriging_job(shape=(36, 36, 8), mark=2, seed=24,
                                                                informed=0.05, max_neighbours=48),
                                                cov_type=W.GAUSSIAN, ranges=(10.0, 10.0, 4.0), nugget=0.02),
}

P_KEYS = ("cov_type", "ranges", "angles", "sill", "nugget", "radii", "max_neighbours")


def _pvec(p):
    return np.array([p["cov_type"], *p["ranges"], *p["angles"], p["sill"], p["nugget"], *p.get("radii", (0, 0, 0)),
                     p.get("max_neighbours", 0)], np.float64)


def _pdict(v):
    return dict(cov_type=int(v[0]), ranges=tuple(v[1:4]), angles=tuple(v[4:7]), sill=float(v[7]),
                nugget=float(v[8]), radii=tuple(int(x) for x in v[9:12]), max_neighbours=int(v[12]))


def load(path):
    z = np.load(path)
    job = {"kind": str(z["kind"]), "shape": tuple(int(v) for v in z["shape"]), "values": z["values"],
           "mask": z["mask"], "secondary_values": z["secondary_values"], "secondary_mask": z["secondary_mask"],
           "params": [_pdict(z["params"])], "primary_mean": float(z["primary_mean"]),
           "secondary_mean": float(z["secondary_mean"]), "correlation": float(z["correlation"])}
    if job["kind"] == "cok1":
        job["secondary_variance"] = float(z["secondary_variance"])
    else:
        job["secondary_cov"] = _pdict(z["secondary_cov"])
    return job, z


def main():
    out_dir = os.path.join(HERE, "cokriging")
    os.makedirs(out_dir, exist_ok=True)
    for name, make in CASES.items():
        job = make()
        out, mask = O.ref_cokriging(job)
        arrays = dict(kind=np.array(job["kind"]), shape=np.array(job["shape"], np.int32), values=job["values"],
                      mask=job["mask"], secondary_values=job["secondary_values"],
                      secondary_mask=job["secondary_mask"], params=_pvec(job["params"][0]),
                      primary_mean=np.float64(job["primary_mean"]), secondary_mean=np.float64(job["secondary_mean"]),
                      correlation=np.float64(job["correlation"]), ref_out=out, ref_mask=mask)
        if job["kind"] == "cok1":
            arrays["secondary_variance"] = np.float64(job["secondary_variance"])
        else:
            arrays["secondary_cov"] = _pvec(job["secondary_cov"])
        np.savez_compressed(os.path.join(out_dir, name + ".npz"), **arrays)
        print(name, "written")


if __name__ == "__main__":
    main()
