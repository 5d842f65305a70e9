"""The reference's own kriging test script on its own test data
(python_pkg/misc/test/test.py:27-120, test_data/NEW_TEST_PROP.INC,
NEW_TEST_PROP_01.INC and mp_0_8_52_55_1.inc; 55x52x1, 143 informed cells),
with the reference's outputs from its sources compiled here
(tests/golden/make_golden_refscript.py writes the fixtures).

* CPU: the oracle restatement gives the reference's outputs, masks and
  per-node lists, weights and variances on every case.
* GPU, through the reference's Python entry points (hpgl_b200.geo_bsd) and
  so through its C ABI (hpgl_ordinary_kriging, hpgl_simple_kriging with a
  given mean and with the automatic mean, hpgl_lvm_kriging, hpgl_median_ik,
  hpgl_indicator_kriging): FP64 outputs and masks bit-identical to the
  reference; mixed precision masks bit-identical and estimates within 1e-6
  relative (floor 1e-6 of the field's scale); per-node neighbour lists bit-
  identical, weights and variances bit-identical (FP64) or within 1e-6
  relative (mixed, floor 1e-6 of the sill).
"""

import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden.make_golden import params_from
from tests.helpers import rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "refscript")
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(FIX, "*.npz")))
REL_TOL = 1e-6


def _load(name):
    z = np.load(os.path.join(FIX, name + ".npz"))
    kind = str(z["kind"])
    job = {"shape": tuple(int(v) for v in z["shape"]), "mask": z["mask"], "params": params_from(z["params"]),
           "kind": kind, "sk_mean": float(z["sk_mean"]), "median_marginal1": float(z["median_marginal1"])}
    for k in ("values", "codes", "mean"):
        if k in z:
            job[k] = z[k]
    return job, kind, bool(z["sk_auto_mean"]), z


def _dump_keys(z, kind, K):
    return [""] if kind != "ik" else ["_c%d" % k for k in range(K)]


def test_fixture_cases_present():
    assert CASES == sorted(["ok", "sk_mean0487", "sk_automatic_mean", "lvm", "median_ik", "ik2", "ik4"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_script(name):
    job, kind, auto, z = _load(name)
    got = O.run(job, kind=kind, sk_auto_mean=auto, dumps=True)
    assert np.array_equal(got["out_mask"], z["ref_mask"])
    if kind in ("ok", "sk", "lvm"):
        assert np.array_equal(got["out"].view(np.uint32), z["ref_out"].view(np.uint32))
    else:
        assert np.array_equal(got["out"], z["ref_out"])
    K = len(job["params"]) if kind == "ik" else 1
    for sfx in _dump_keys(z, kind, K):
        if "sample" + sfx not in z:
            continue
        k = int(sfx[2:]) if sfx else 0
        slots = z["sample" + sfx].astype(np.int64) * K + k
        cap = got["cap"]
        assert np.array_equal(got["nb_count"][slots], z["ref_nb_count" + sfx])
        assert np.array_equal(got["status"][slots], z["ref_status" + sfx])
        n = z["ref_nb_count" + sfx]
        valid = np.arange(z["ref_nb_index" + sfx].shape[1])[None, :] < n[:, None]
        gi = got["nb_index"].reshape(-1, cap)[slots][:, :valid.shape[1]]
        assert np.array_equal(gi[valid], z["ref_nb_index" + sfx][valid])
        gw = got["weights"].reshape(-1, cap)[slots][:, :valid.shape[1]]
        assert np.array_equal(gw[valid].view(np.uint64), z["ref_weights" + sfx][valid].view(np.uint64))
        ok = z["ref_status" + sfx] == 0
        assert np.array_equal(got["variance"][slots][ok].view(np.uint64),
                              z["ref_variance" + sfx][ok].view(np.uint64))


def _cov(geo, p):
    return geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], angles=p["angles"], sill=p["sill"],
                               nugget=p["nugget"])


def _run_entry(name, precision):
    """The case through the reference's Python entry point that the script calls."""
    from hpgl_b200.geo_bsd import geo
    job, kind, auto, z = _load(name)
    grid = geo.SugarboxGrid(*job["shape"])
    p = job["params"][0]
    if kind in ("ok", "sk", "lvm"):
        prop = geo.ContProperty(job["values"].copy(), job["mask"].copy())
        if kind == "ok":
            out = geo.ordinary_kriging(prop, grid, p["radii"], p["max_neighbours"], _cov(geo, p), precision=precision)
        elif kind == "sk":
            mean = None if auto else job["sk_mean"]
            out = geo.simple_kriging(prop, grid, p["radii"], p["max_neighbours"], _cov(geo, p), mean=mean,
                                     precision=precision)
        else:
            out = geo.lvm_kriging(prop, grid, job["mean"], p["radii"], p["max_neighbours"], _cov(geo, p),
                                  precision=precision)
        return out, z, kind
    K = len(job["params"]) if kind == "ik" else 2
    prop = geo.IndProperty(job["codes"].copy(), job["mask"].copy(), K)
    if kind == "median_ik":
        m1 = job["median_marginal1"]
        out = geo.median_ik(prop, grid, (1.0 - m1, m1), p["radii"], p["max_neighbours"], _cov(geo, p),
                            precision=precision)
    elif K == 2:
        # geo.indicator_kriging routes two categories to median IK; the
        # full two-category indicator kriging is the C ABI's own
        import ctypes as C
        from hpgl_b200.geo_bsd.hpgl_wrap import check_last_error
        out = geo._clone_prop(prop)
        data = [dict(cov_model=_cov(geo, q), radiuses=q["radii"], max_neighbours=q["max_neighbours"])
                for q in job["params"]]
        params = geo._ik_params(data, [q["marginal_prob"] for q in job["params"]])
        inp, outp = geo._ind_array(prop, grid), geo._ind_array(out, grid)
        with geo._Precision(precision):
            geo._hpgl_so.hpgl_indicator_kriging(C.byref(inp), C.byref(outp), params, K)
            check_last_error()
    else:
        data = [dict(cov_model=_cov(geo, q), radiuses=q["radii"], max_neighbours=q["max_neighbours"])
                for q in job["params"]]
        out = geo.indicator_kriging(prop, grid, data, [q["marginal_prob"] for q in job["params"]],
                                    precision=precision)
    return out, z, kind


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", CASES)
def test_reference_script_entry_points(native_lib, name, precision):
    out, z, kind = _run_entry(name, precision)
    data = out.data.reshape(-1, order="F")
    mask = out.mask.reshape(-1, order="F")
    assert np.array_equal(mask, z["ref_mask"])
    if kind in ("ok", "sk", "lvm"):
        if precision == "fp64":
            assert np.array_equal(data.view(np.uint32), z["ref_out"].view(np.uint32))
        else:
            informed = z["mask"] > 0
            scale = float(np.max(np.abs(z["values"][informed])))
            assert rel_err(data, z["ref_out"], 1e-6 * scale).max() <= REL_TOL
    else:
        assert np.array_equal(data, z["ref_out"])


def test_two_category_geo_routes_to_median():
    """geo.indicator_kriging with the script's two-category ik_data runs
    median IK (geo.py:493-501): the fixtures' parameters agree."""
    j2, _, _, _ = _load("ik2")
    jm, _, _, _ = _load("median_ik")
    q = dict(j2["params"][0])
    q.pop("marginal_prob")
    r = dict(jm["params"][0])
    r.pop("marginal_prob")
    assert q == r
    assert 1.0 - j2["params"][0]["marginal_prob"] == jm["median_marginal1"]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", [c for c in CASES if c != "sk_automatic_mean"])
def test_reference_script_per_node(native_lib, name, precision):
    from hpgl_b200 import native as N
    job, kind, auto, z = _load(name)
    got = N.krige(job, precision=precision, kind=kind, dumps=True, sk_auto_mean=auto)
    K = len(job["params"]) if kind == "ik" else 1
    # categories with identical variograms and searches share one system per
    # node: the library then keeps one slot per node
    Kg = len(got["status"]) // int(np.prod(job["shape"]))
    sill = max(q["sill"] for q in job["params"])
    for sfx in _dump_keys(z, kind, K):
        k = int(sfx[2:]) if sfx else 0
        slots = z["sample" + sfx].astype(np.int64) * Kg + (k if Kg > 1 else 0)
        cap = got["cap"]
        n = z["ref_nb_count" + sfx]
        assert np.array_equal(got["nb_count"][slots], n)
        assert np.array_equal(got["status"][slots], z["ref_status" + sfx])
        valid = np.arange(z["ref_nb_index" + sfx].shape[1])[None, :] < n[:, None]
        gi = got["nb_index"].reshape(-1, cap)[slots][:, :valid.shape[1]]
        assert np.array_equal(gi[valid], z["ref_nb_index" + sfx][valid])
        ok = z["ref_status" + sfx] == 0
        gw = got["weights"].reshape(-1, cap)[slots][:, :valid.shape[1]]
        gv = got["variance"][slots]
        if precision == "fp64":
            assert np.array_equal(gw[valid].view(np.uint64), z["ref_weights" + sfx][valid].view(np.uint64))
            assert np.array_equal(gv[ok].view(np.uint64), z["ref_variance" + sfx][ok].view(np.uint64))
        else:
            assert rel_err(gw[valid], z["ref_weights" + sfx][valid], 1e-6).max() <= REL_TOL
            assert rel_err(gv[ok], z["ref_variance" + sfx][ok], 1e-6 * sill).max() <= REL_TOL
