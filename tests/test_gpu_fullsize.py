"""Full-size benchmark configurations on the GPU, checked against the CPU
oracle on a seeded sample of nodes (the oracle searches the whole grid but
solves only the sampled nodes):

* 256x256x64 SK and OK (exponential, azimuth 30, 32 neighbours)
* 200x200x100 4-category IK (24 neighbours)
* 512x512x32 LVM (Gaussian, clustered data, 64 neighbours; mixes the
  template and clusterizer searches and has singular systems)

Neighbour lists, statuses and masks must be bit-identical; estimates are
bit-identical on the FP64 path and within 1e-6 relative on the mixed path.
Size-independent checks on the whole grid: every uninformed node is either
kriged (mask 1) or, for OK, left as the input; informed nodes are copied.
"""

import numpy as np
import pytest

from hpgl_b200 import native as N
from hpgl_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import rel_err

SAMPLE = 1500

CONFIGS = {
    "sk_256x256x64": (W.sk_ok_256x256x64, "sk"),
    "ok_256x256x64": (W.sk_ok_256x256x64, "ok"),
    "ik_200x200x100": (W.ik_200x200x100, "ik"),
    "lvm_512x512x32": (W.lvm_512x512x32, "lvm"),
}

_jobs = {}


def _job(name):
    if name not in _jobs:
        make, kind = CONFIGS[name]
        job = make()
        size = int(np.prod(job["shape"]))
        rng = np.random.default_rng(2024)
        pool = np.arange(size) if kind == "ik" else np.nonzero(job["mask"] == 0)[0]
        sample = np.sort(rng.choice(pool, SAMPLE, replace=False)).astype(np.int32)
        ref = O.run(job, kind=kind, node_list=sample)
        _jobs[name] = (job, kind, sample, ref)
    return _jobs[name]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CONFIGS))
def test_fullsize_sampled_parity(native_lib, name, precision):
    job, kind, sample, ref = _job(name)
    got = N.krige(job, precision=precision, kind=kind, dumps=True)
    K = len(job["params"]) if kind == "ik" else 1
    sr = sample.astype(np.int64) * K
    sg = sample.astype(np.int64)
    assert np.array_equal(ref["status"][sr], got["status"][sg])
    cap = ref["cap"]
    assert np.array_equal(ref["nb_count"][sr], got["nb_count"][sg])
    ri = ref["nb_index"].reshape(-1, cap)[sr]
    gi = got["nb_index"].reshape(-1, got["cap"])[sg][:, :cap]
    valid = np.arange(cap)[None, :] < ref["nb_count"][sr][:, None]
    assert np.array_equal(ri[valid], gi[valid]), "neighbour lists differ"
    assert np.array_equal(ref["out_mask"][sample], got["out_mask"][sample])
    if kind == "ik":
        assert np.array_equal(ref["out"][sample], got["out"][sample])
    elif precision == "fp64":
        assert np.array_equal(ref["out"][sample].view(np.uint32), got["out"][sample].view(np.uint32))
    else:
        informed = job["mask"] > 0
        scale = float(np.max(np.abs(job["values"][informed])))
        assert rel_err(got["out"][sample], ref["out"][sample], 1e-6 * scale).max() <= 1e-6
    ok = ref["status"][sr] == 0
    rv, gv = ref["variance"][sr][ok], got["variance"][sg][ok]
    if precision == "fp64":
        assert np.array_equal(rv.view(np.uint64), gv.view(np.uint64)), "variances differ"
    else:
        sill = job["params"][0]["sill"]
        assert rel_err(gv, rv, 1e-6 * sill).max() <= 1e-6, "variances beyond 1e-6"
    # whole-grid properties
    if kind in ("sk", "lvm", "ik"):
        assert got["out_mask"].all(), "every node is written"
    if kind in ("ok", "sk", "lvm"):
        informed = job["mask"] > 0
        assert np.array_equal(got["out"][informed].view(np.uint32), job["values"][informed].view(np.uint32))
    if precision == "mixed":
        assert got["systems_fp64"] <= got["systems"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CONFIGS))
def test_fullsize_mixed_against_fp64_whole_grid(native_lib, name):
    """Every node of the full-size configuration: the mixed path (FP32
    factorisation + FP64 refinement, FP64 re-solve of routed systems)
    against the FP64 path (bit-identical to the oracle on the sampled
    nodes): statuses and masks identical; estimates within 1e-6 relative
    (floor 1e-6 of the field's scale), variances within 1e-6 relative
    (floor 1e-6 of the sill); IK categories identical."""
    job, kind, _, _ = _job(name)
    ref = N.krige(job, precision="fp64", kind=kind, dumps="variance")
    got = N.krige(job, precision="mixed", kind=kind, dumps="variance")
    assert np.array_equal(ref["status"], got["status"])
    assert np.array_equal(ref["out_mask"], got["out_mask"])
    if kind == "ik":
        assert np.array_equal(ref["out"], got["out"])
    else:
        informed = job["mask"] > 0
        scale = float(np.max(np.abs(job["values"][informed])))
        assert rel_err(got["out"], ref["out"], 1e-6 * scale).max() <= 1e-6
    ok = ref["status"] == 0
    sill = job["params"][0]["sill"]
    assert rel_err(got["variance"][ok], ref["variance"][ok], 1e-6 * sill).max() <= 1e-6
