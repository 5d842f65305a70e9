"""Loader of the simulation fixtures (tests/golden/sim/, made from the
compiled reference by tests/golden/make_golden_sim.py)."""

import glob
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sim")


def paths(kind):
    return sorted(glob.glob(os.path.join(GOLDEN, kind + "_*.npz")))


def load(path):
    z = np.load(path)
    d = {k: z[k] for k in z.files}
    d["shape"] = tuple(int(v) for v in d["shape"])
    d["params"] = json.loads(str(d["params"]))
    for p in d["params"]:
        for k in ("ranges", "angles", "radii"):
            p[k] = tuple(p[k])
    d["seed"] = int(d["seed"])
    return d


def sgs_kwargs(d):
    kw = dict(seed=d["seed"], ordinary=bool(d["ordinary"]))
    if "lvm" in d:
        kw["lvm"] = d["lvm"]
    if "sim_mask" in d:
        kw["sim_mask"] = d["sim_mask"]
    if "cdf_values" in d:
        kw["cdf"] = (d["cdf_values"], d["cdf_probs"])
    return kw
