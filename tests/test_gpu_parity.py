"""GPU parity against the CPU oracle (the reference algorithm restated in
oracle/hpgl_oracle.cpp, itself pinned to the compiled reference).

FP64 path: neighbour lists, statuses, masks, estimates, variances and weights
are bit-identical to the oracle's.  Mixed path (FP32 factorisation + FP64
refinement): neighbour lists, statuses and masks bit-identical; estimates and
variances within 1e-6 relative (floor 1e-6 of the field's scale).
"""

import numpy as np
import pytest

from hpgl_b200 import native as N
from hpgl_b200 import workloads as W
from oracle import oracle as O
from tests.helpers import f32_bits_equal, neighbour_lists_equal, rel_err

REL_TOL = 1e-6

CASES = {
    "ok_50x50x20": (lambda: W.ok_50x50x20(), "ok"),
    "sk_64x64x32": (lambda: W.sk_ok_256x256x64(shape=(64, 64, 32)), "sk"),
    "ok_64x64x32": (lambda: W.sk_ok_256x256x64(shape=(64, 64, 32)), "ok"),
    "ik_50x50x25": (lambda: W.ik_200x200x100(shape=(50, 50, 25)), "ik"),
    "median_ik_50x50x25": (lambda: W.ik_200x200x100(shape=(50, 50, 25)), "median_ik"),
    "lvm_96x96x16": (lambda: W.lvm_512x512x32(shape=(96, 96, 16)), "lvm"),
}



def _nmax(job, n, **over):
    """The same job searching up to n neighbours (33..64: the wide solves)."""
    job = dict(job)
    job["params"] = [dict(p, max_neighbours=n, **over) for p in job["params"]]
    return job


# Systems of 33 to 64 neighbours, every kind, ragged counts near sparse
# regions and the grid's edges; the long-range Gaussian model without nugget
# makes the systems ill-conditioned (about 1.5 % fail the FP64 factorisation,
# FP32 pivots are routed to the FP64 re-solve).
CASES.update({
    "ok_n48_48x48x24": (lambda: _nmax(W.sk_ok_256x256x64(shape=(48, 48, 24)), 48), "ok"),
    "sk_n64_48x48x24": (lambda: _nmax(W.sk_ok_256x256x64(shape=(48, 48, 24)), 64), "sk"),
    "ik_n40_40x40x20": (lambda: _nmax(W.ik_200x200x100(shape=(40, 40, 20)), 40), "ik"),
    "median_ik_n56_40x40x20": (lambda: _nmax(W.ik_200x200x100(shape=(40, 40, 20)), 56), "median_ik"),
    "ok_gauss_n64_48x48x16": (lambda: _nmax(W.lvm_512x512x32(shape=(48, 48, 16)), 64, nugget=0.0,
                                            ranges=(300.0, 300.0, 40.0)), "ok"),
})

_cache = {}


def _oracle(name):
    if name not in _cache:
        make, kind = CASES[name]
        job = make()
        _cache[name] = (job, kind, O.run(job, kind=kind))
    return _cache[name]


def _slots(job, kind, ref):
    """(oracle slots, gpu slots) of kriged systems: IK with identical
    categories keeps one GPU slot per node vs the oracle's node*K + k."""
    size = int(np.prod(job["shape"]))
    if kind == "ik":
        K = len(job["params"])
        nodes = np.arange(size)
        return nodes * K, nodes
    s = np.nonzero(ref["status"] >= 0)[0]
    return s, s


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CASES))
def test_parity(native_lib, name, precision):
    job, kind, ref = _oracle(name)
    got = N.krige(job, precision=precision, kind=kind, dumps=True)
    sr, sg = _slots(job, kind, ref)
    assert np.array_equal(ref["out_mask"], got["out_mask"]), "mask differs"
    assert np.array_equal(ref["status"][sr], got["status"][sg]), "status differs"
    ok, msg = neighbour_lists_equal(ref, got, sr, sg, ref["cap"], got["cap"])
    assert ok, msg
    solved = ref["status"][sr] == 0
    if kind in ("ok", "sk", "lvm"):
        if precision == "fp64":
            assert f32_bits_equal(ref["out"], got["out"]), "estimates differ"
        else:
            scale = float(np.max(np.abs(ref["out"][ref["out_mask"] > 0])))
            e = rel_err(got["out"], ref["out"], 1e-6 * scale)
            assert e.max() <= REL_TOL, "estimate rel err %g" % e.max()
    else:
        assert np.array_equal(ref["out"], got["out"]), "categories differ"
    rv, gv = ref["variance"][sr][solved], got["variance"][sg][solved]
    if precision == "fp64":
        assert np.array_equal(rv.view(np.uint64), gv.view(np.uint64)), "variances differ"
        cap = ref["cap"]
        rw = ref["weights"].reshape(-1, cap)[sr][solved]
        gw = got["weights"].reshape(-1, got["cap"])[sg][solved][:, :cap]
        cnt = ref["nb_count"][sr][solved]
        valid = np.arange(cap)[None, :] < cnt[:, None]
        assert np.array_equal(rw[valid].view(np.uint64), gw[valid].view(np.uint64)), "weights differ"
    else:
        e = rel_err(gv, rv, 1e-6 * float(np.max(np.abs(rv))))
        assert e.max() <= REL_TOL, "variance rel err %g" % e.max()
