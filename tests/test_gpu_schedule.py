"""Launch schedules and the autotuner.

The fused kernel (template search + solve in one persistent launch) and the
separate search and solve kernels run the same per-node code.  In FP64 every
output -- estimates, masks, statuses, neighbour lists, weights, variances --
is bit-identical under both, for every block count.  In mixed precision the
masks, statuses and neighbour lists are identical and the values agree
within twice the mixed tolerance (each is within 1e-6 of FP64): which
systems a warp sends
straight to the FP64 re-solve depends on the nodes that warp met before
(the per-warp routing guess), and so on the schedule.  hpgl_b200_autotune
tries the candidates and leaves the fastest in force without changing any
result."""

import numpy as np
import pytest

from hpgl_b200 import native as N
from hpgl_b200 import workloads as W
from tests.helpers import rel_err

JOBS = {
    "ok_n12": (lambda: W.ok_50x50x20(), "ok", 0),
    "sk_n32": (lambda: W.sk_ok_256x256x64(shape=(48, 48, 24)), "sk", 0),
    "lvm_n64": (lambda: W.lvm_512x512x32(shape=(64, 64, 12)), "lvm", 1),
    "ik_n24": (lambda: W.ik_200x200x100(shape=(36, 36, 18)), "ik", 0),
}

def _bits(x):
    return np.ascontiguousarray(x).tobytes()


def _same(a, b):
    """Name of the first output that differs (defined entries only: variance
    and weights of solved slots, the first count entries of each list)."""
    for k in ("out", "out_mask", "status", "nb_count"):
        if _bits(a[k]) != _bits(b[k]):
            return k
    cap = a["cap"]
    solved = a["status"] == 0
    if _bits(a["variance"][solved]) != _bits(b["variance"][solved]):
        return "variance"
    valid = np.arange(cap)[None, :] < a["nb_count"][:, None]
    ia, ib = a["nb_index"].reshape(-1, cap), b["nb_index"].reshape(-1, cap)
    if _bits(ia[valid]) != _bits(ib[valid]):
        return "nb_index"
    wa, wb = a["weights"].reshape(-1, cap), b["weights"].reshape(-1, cap)
    wv = valid & solved[:, None]
    if _bits(wa[wv]) != _bits(wb[wv]):
        return "weights"
    return None


@pytest.fixture(autouse=True)
def _restore_default():
    yield
    for fam in (0, 1):
        for prec in ("fp64", "mixed"):
            N.set_launch(fam, prec, "split", 0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(JOBS))
def test_split_and_fused_agree(native_lib, name, precision):
    make, kind, fam = JOBS[name]
    job = make()
    runs = []
    for sched, bps in (("split", 0), ("fused", 0), ("fused", 1)):
        N.set_launch(fam, precision, sched, bps)
        runs.append(N.krige(job, precision=precision, kind=kind, dumps=True))
    for r in runs[1:]:
        _agree(runs[0], r, job, kind, precision)


def _agree(a, r, job, kind, precision):
    """FP64: bit-identical; mixed: identical masks, statuses and lists,
    values within twice the mixed tolerance."""
    if precision == "fp64":
        k = _same(a, r)
        assert k is None, "%s differs between schedules" % k
        return
    for k in ("out_mask", "status", "nb_count"):
        assert _bits(a[k]) == _bits(r[k]), "%s differs between schedules" % k
    solved = a["status"] == 0
    if kind == "ik":
        assert _bits(a["out"]) == _bits(r["out"])
    else:
        scale = float(np.max(np.abs(job["values"][job["mask"] > 0])))
        assert rel_err(r["out"], a["out"], 1e-6 * scale).max() <= 2e-6
    sill = job["params"][0]["sill"]
    assert rel_err(r["variance"][solved], a["variance"][solved], 1e-6 * sill).max() <= 2e-6


@pytest.mark.gpu
def test_autotune_keeps_results(native_lib):
    job = W.sk_ok_256x256x64(shape=(64, 64, 32))
    before = N.krige(job, precision="mixed", kind="sk", dumps=True)
    t = N.autotune(job, precision="mixed", kind="sk")
    assert len(t["candidates"]) >= 2
    assert {c["schedule"] for c in t["candidates"]} == {"split", "fused"}
    assert all(c["ms"] > 0 for c in t["candidates"])
    assert t["chosen"]["ms"] == min(c["ms"] for c in t["candidates"])
    after = N.krige(job, precision="mixed", kind="sk", dumps=True)
    _agree(before, after, job, "sk", "mixed")
