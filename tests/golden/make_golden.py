"""Generates the golden fixtures of the kriging path from the reference's own
sources compiled by oracle/build_ref.sh (oracle/_ref/libhpgl_ref.so): for
small seeded inputs of every kind, the reference's C-ABI outputs (estimate or
category, mask) and, from the dump driver oracle/ref_dump.cpp, per-node
neighbour lists, weights, variances and statuses.

    python tests/golden/make_golden.py      # needs the reference checkout

Writes tests/golden/<case>.npz (inputs included, so the fixtures do not
depend on numpy's RNG staying the same)."""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hpgl_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    "ok_spherical_24x20x10": (lambda: W.ok_50x50x20(shape=(24, 20, 10), seed=11), "ok"),
    "sk_exponential_az30_32x32x12": (lambda: W.sk_ok_256x256x64(shape=(32, 32, 12), seed=12), "sk"),
    "ok_exponential_az30_32x32x12": (lambda: W.sk_ok_256x256x64(shape=(32, 32, 12), seed=12), "ok"),
    "lvm_gaussian_blobs_40x40x8": (lambda: W.lvm_512x512x32(shape=(40, 40, 8), seed=14, blobs=6), "lvm"),
    "ik4_spherical_24x24x10": (lambda: W.ik_200x200x100(shape=(24, 24, 10), seed=13), "ik"),
    "median_ik_24x24x10": (lambda: W.ik_200x200x100(shape=(24, 24, 10), seed=15, categories=2), "median_ik"),
}


def job_arrays(job, kind):
    out = {"shape": np.array(job["shape"], np.int32), "mask": job["mask"]}
    for k in ("values", "codes", "mean"):
        if k in job:
            out[k] = job[k]
    p = job["params"]
    out["params"] = np.array([[q["cov_type"], *q["ranges"], *q["angles"], q["sill"], q["nugget"], *q["radii"],
                               q["max_neighbours"], q["marginal_prob"]] for q in p], np.float64)
    out["kind"] = np.array(kind)
    return out


def params_from(arr):
    ps = []
    for r in arr:
        ps.append(dict(cov_type=int(r[0]), ranges=tuple(r[1:4]), angles=tuple(r[4:7]), sill=float(r[7]),
                       nugget=float(r[8]), radii=tuple(int(v) for v in r[9:12]), max_neighbours=int(r[12]),
                       marginal_prob=float(r[13])))
    return ps


def load(path):
    z = np.load(path)
    kind = str(z["kind"])
    job = {"shape": tuple(int(v) for v in z["shape"]), "mask": z["mask"], "params": params_from(z["params"]),
           "kind": kind, "sk_mean": 0.0}
    for k in ("values", "codes", "mean"):
        if k in z:
            job[k] = z[k]
    if kind == "median_ik":
        job["median_marginal1"] = 0.5
    return job, kind, z


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref/libhpgl_ref.so not built (oracle/build_ref.sh)")
    for name, (make, kind) in CASES.items():
        job = make()
        if kind == "median_ik":
            job["median_marginal1"] = 0.5
        out, mask = O.ref_run(job, kind=kind)
        arrays = job_arrays(job, kind)
        arrays["ref_out"] = out
        arrays["ref_mask"] = mask
        if kind == "ik":
            d = O.ref_dump(job, kind=kind, category=0)
        else:
            d = O.ref_dump(job, kind=kind)
        # per-node dumps for a seeded sample of the kriged nodes (kept small)
        kriged = np.nonzero(d["status"] >= 0)[0]
        rng = np.random.default_rng(99)
        sample = np.sort(rng.choice(kriged, min(256, len(kriged)), replace=False)).astype(np.int32)
        arrays["sample"] = sample
        arrays["ref_nb_count"] = d["nb_count"][sample]
        arrays["ref_nb_index"] = d["nb_index"].reshape(-1, d["cap"])[sample]
        arrays["ref_weights"] = d["weights"].reshape(-1, d["cap"])[sample]
        arrays["ref_variance"] = d["variance"][sample]
        arrays["ref_status"] = d["status"][sample]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        print("wrote", name, os.path.getsize(os.path.join(HERE, name + ".npz")), "bytes")


if __name__ == "__main__":
    main()
