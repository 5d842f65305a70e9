"""Colocated simple cokriging (Markov models I and II) on the GPU against the
oracle and the reference's golden fixtures: estimates, masks, statuses,
neighbour lists and the N+1 weights of every node bit for bit (the GPU path
runs the reference's gauss_solve in its own operation order), including
nodes without neighbours (the failure estimate m1 + s - m2) and
ill-conditioned Gaussian systems; and the drop-in entry points
simple_cokriging_markI / simple_cokriging_markII."""

import glob
import os

import numpy as np
import pytest

from hpgl_b200 import native as N
from hpgl_b200 import workloads as W
from oracle import oracle as O
from tests.golden.make_golden_cokriging import CASES, load

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "cokriging", "*.npz")))


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.tobytes()


def _compare(ref, got):
    assert _bits(ref["out"]) == _bits(got["out"]), "estimates differ"
    assert np.array_equal(ref["out_mask"], got["out_mask"]), "masks differ"
    assert np.array_equal(ref["status"], got["status"]), "statuses differ"
    assert np.array_equal(ref["nb_count"], got["nb_count"]), "neighbour counts differ"
    cr, cg = ref["cap"], got["cap"]  # oracle: lists of max_neighbours; GPU: one longer (weights)
    cnt = ref["nb_count"]
    valid = np.arange(cr)[None, :] < cnt[:, None]
    ri = ref["nb_index"].reshape(-1, cr)
    gi = got["nb_index"].reshape(-1, cg)[:, :cr]
    assert np.array_equal(ri[valid], gi[valid]), "neighbour lists differ"
    solved = ref["status"] == 0
    wv = (np.arange(cr + 1)[None, :] <= cnt[:, None]) & solved[:, None]
    rw = ref["weights"].reshape(-1, cr + 1)
    gw = got["weights"].reshape(-1, cg)
    assert _bits(rw[wv]) == _bits(gw[wv]), "weights differ"


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_cokriging_parity(native_lib, name):
    job = CASES[name]()
    ref = O.cokriging(job)
    got = N.krige(job, dumps=True)
    _compare(ref, got)


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_cokriging_golden(native_lib, path):
    job, z = load(path)
    got = N.krige(job)
    assert _bits(got["out"]) == _bits(z["ref_out"]), "estimates differ from the reference's"
    assert np.array_equal(got["out_mask"], z["ref_mask"])


@pytest.mark.gpu
def test_cokriging_larger_grid(native_lib):
    job = W.cokriging_job(shape=(96, 96, 24), mark=2, seed=31, max_neighbours=64)
    ref = O.cokriging(job)
    got = N.krige(job, dumps=True)
    _compare(ref, got)


@pytest.mark.gpu
def test_cokriging_dropin_entry_points(native_lib):
    from hpgl_b200.geo_bsd import geo
    for mark in (1, 2):
        job = W.cokriging_job(shape=(36, 30, 8), mark=mark, seed=50 + mark)
        ref = O.cokriging(job)
        grid = geo.SugarboxGrid(*job["shape"])
        shape = job["shape"]

        def prop(values, mask):
            return geo.ContProperty(np.asfortranarray(values.reshape(shape, order="F")),
                                    np.asfortranarray(mask.reshape(shape, order="F")))
        primary = prop(job["values"], job["mask"])
        secondary = prop(job["secondary_values"], job["secondary_mask"])
        p = job["params"][0]
        cm = geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], angles=p["angles"], sill=p["sill"],
                                 nugget=p["nugget"])
        if mark == 1:
            out = geo.simple_cokriging_markI(primary, grid, secondary, job["primary_mean"], job["secondary_mean"],
                                             job["secondary_variance"], job["correlation"], p["radii"],
                                             p["max_neighbours"], cm)
        else:
            s = job["secondary_cov"]
            scm = geo.CovarianceModel(type=s["cov_type"], ranges=s["ranges"], angles=s["angles"], sill=s["sill"],
                                      nugget=s["nugget"])
            out = geo.simple_cokriging_markII(grid, {"data": primary, "mean": job["primary_mean"], "cov_model": cm},
                                              {"data": secondary, "mean": job["secondary_mean"], "cov_model": scm},
                                              job["correlation"], p["radii"], p["max_neighbours"])
        vals = np.asarray(out.data).reshape(-1, order="F")
        mask = np.asarray(out.mask).reshape(-1, order="F")
        assert _bits(vals.astype(np.float32)) == _bits(ref["out"]), "mark %d estimates differ" % mark
        assert np.array_equal(mask.astype(np.uint8), ref["out_mask"])
