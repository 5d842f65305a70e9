"""The reference's Python entry points (hpgl_b200.geo_bsd, names and
arguments of geo_bsd/geo.py) on the GPU, against the oracle, including the
boundary's output semantics: outputs start as a copy of the input, ordinary
kriging leaves nodes without neighbours untouched, SK/LVM write the mean
there, indicator kriging with 2 categories routes to median IK."""

import numpy as np
import pytest

from hpgl_b200 import workloads as W
from oracle import oracle as O


def _cont_prop(job):
    from hpgl_b200.geo_bsd import geo
    return geo.ContProperty(job["values"], job["mask"])


@pytest.mark.gpu
def test_ordinary_kriging_entry(native_lib):
    from hpgl_b200.geo_bsd import geo
    job = W.ok_50x50x20(shape=(30, 30, 10), seed=7)
    p = job["params"][0]
    cm = geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], angles=p["angles"], sill=p["sill"],
                             nugget=p["nugget"])
    out = geo.ordinary_kriging(_cont_prop(job), geo.SugarboxGrid(30, 30, 10), p["radii"], p["max_neighbours"], cm)
    ref = O.run(job, dumps=False)
    assert np.array_equal(out.mask.reshape(-1, order="F"), ref["out_mask"])
    assert np.array_equal(out.data.reshape(-1, order="F").view(np.uint32), ref["out"].view(np.uint32))
    mixed = geo.ordinary_kriging(_cont_prop(job), geo.SugarboxGrid(30, 30, 10), p["radii"], p["max_neighbours"], cm,
                                 precision="mixed")
    assert np.array_equal(mixed.mask.reshape(-1, order="F"), ref["out_mask"])


def _isolated_job():
    # informed cells only in one corner: far nodes find no neighbour
    nx, ny, nz = 40, 40, 1
    values = np.full(nx * ny * nz, -99.0, np.float32)
    mask = np.zeros(nx * ny * nz, np.uint8)
    rng = np.random.default_rng(5)
    for _ in range(30):
        x, y = rng.integers(0, 8, 2)
        i = x + nx * y
        mask[i] = 1
        values[i] = rng.standard_normal()
    p = W.cov_params(0, (6, 6, 6), radii=(6, 6, 1), max_neighbours=8)
    return dict(shape=(nx, ny, nz), values=values, mask=mask, params=[p], sk_mean=0.25,
                mean=np.linspace(-1, 1, nx * ny * nz).astype(np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ok", "sk", "lvm"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_failure_semantics(native_lib, kind, precision):
    from hpgl_b200 import native as N
    job = _isolated_job()
    ref = O.run(job, kind=kind, dumps=True)
    assert (ref["status"] == 1).sum() > 100, "case must contain nodes without neighbours"
    got = N.krige(job, precision=precision, kind=kind, dumps=True)
    assert np.array_equal(got["status"], ref["status"])
    assert np.array_equal(got["out_mask"], ref["out_mask"])
    assert np.array_equal(got["out"].view(np.uint32), ref["out"].view(np.uint32))
    if kind == "ok":
        untouched = ref["status"] == 1
        assert (got["out_mask"][untouched] == 0).all()
        assert (got["out"][untouched] == -99.0).all()


@pytest.mark.gpu
def test_indicator_entry_points(native_lib):
    from hpgl_b200.geo_bsd import geo
    job = W.ik_200x200x100(shape=(24, 24, 10), seed=21)
    p = job["params"][0]
    cm = geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], sill=p["sill"], nugget=p["nugget"])
    prop = geo.IndProperty(job["codes"], job["mask"], 4)
    data = [dict(cov_model=cm, radiuses=p["radii"], max_neighbours=p["max_neighbours"]) for _ in range(4)]
    out = geo.indicator_kriging(prop, geo.SugarboxGrid(24, 24, 10), data, [0.25] * 4)
    ref = O.run(job, kind="ik", dumps=False)
    assert np.array_equal(out.data.reshape(-1, order="F"), ref["out"])
    assert out.mask.all()
    # two categories route to median IK with marginal probabilities (p0, 1 - p0)
    job2 = W.ik_200x200x100(shape=(24, 24, 10), seed=22, categories=2)
    prop2 = geo.IndProperty(job2["codes"], job2["mask"], 2)
    data2 = [dict(cov_model=cm, radiuses=p["radii"], max_neighbours=p["max_neighbours"]) for _ in range(2)]
    out2 = geo.indicator_kriging(prop2, geo.SugarboxGrid(24, 24, 10), data2, [0.6, 0.4])
    ref2 = O.run(dict(job2, median_marginal1=0.4), kind="median_ik", dumps=False)
    assert np.array_equal(out2.data.reshape(-1, order="F"), ref2["out"])


@pytest.mark.gpu
def test_ik_with_differing_categories(native_lib):
    from hpgl_b200 import native as N
    job = W.ik_200x200x100(shape=(24, 24, 10), seed=23, categories=3)
    job["params"][1] = dict(job["params"][1], ranges=(15.0, 15.0, 4.0), radii=(15, 15, 4), max_neighbours=16)
    job["params"][2] = dict(job["params"][2], cov_type=1, marginal_prob=0.5)
    ref = O.run(job, kind="ik", dumps=True)
    got = N.krige(job, precision="fp64", kind="ik", dumps=True)
    assert np.array_equal(got["out"], ref["out"])
    assert np.array_equal(got["status"], ref["status"])
    assert np.array_equal(got["probs"].view(np.uint32), ref["probs"].view(np.uint32))


def _sk_params(p, automatic, mean):
    from hpgl_b200.geo_bsd import geo
    from hpgl_b200.geo_bsd.hpgl_wrap import _HPGL_SK_PARAMS
    cm = geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], angles=p["angles"], sill=p["sill"],
                             nugget=p["nugget"])
    return _HPGL_SK_PARAMS(automatic_mean=int(automatic), mean=mean,
                           **geo._kriging_fields(cm, p["radii"], p["max_neighbours"]))


@pytest.mark.gpu
@pytest.mark.parametrize("automatic", [False, True])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_simple_kriging_c_abi(native_lib, automatic, precision):
    """hpgl_simple_kriging (api.cpp:261-288) called with the reference's
    struct: a given mean, or m_automatic_mean = 1 -- the mean of the
    informed values (calc_mean.cpp:6-30, simple_kriging.cpp:50-59), the
    given mean ignored."""
    import ctypes as C
    from hpgl_b200.geo_bsd import geo
    from hpgl_b200.geo_bsd.hpgl_wrap import check_last_error
    from tests.helpers import rel_err
    job = W.sk_ok_256x256x64(shape=(40, 40, 16), seed=41)
    job["values"] = (job["values"] + np.where(job["mask"] > 0, 0.75, 0.0)).astype(np.float32)
    job["sk_mean"] = 0.3
    p = job["params"][0]
    skp = _sk_params(p, automatic, 0.3)
    data = np.require(job["values"].copy(), np.float32, "F")
    mask = np.require(job["mask"].copy(), np.uint8, "F")
    out, out_mask = data.copy(), mask.copy()
    sh = geo._create_hpgl_shape(job["shape"])
    with geo._Precision(precision):
        geo._hpgl_so.hpgl_simple_kriging(data, mask, C.byref(sh), C.byref(skp), out, out_mask, C.byref(sh))
        check_last_error()
    ref = O.run(job, kind="sk", sk_auto_mean=automatic, dumps=False)
    other = O.run(job, kind="sk", sk_auto_mean=not automatic, dumps=False)
    assert not np.array_equal(ref["out"], other["out"]), "the two means must give different estimates"
    assert np.array_equal(out_mask, ref["out_mask"])
    if precision == "fp64":
        assert np.array_equal(out.view(np.uint32), ref["out"].view(np.uint32))
    else:
        scale = float(np.max(np.abs(job["values"][job["mask"] > 0])))
        assert rel_err(out, ref["out"], 1e-6 * scale).max() <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_simple_kriging_entry_without_mean(native_lib, precision):
    """geo.simple_kriging(..., mean=None) (geo.py:402-425) krigs with the
    automatic mean."""
    from hpgl_b200.geo_bsd import geo
    from tests.helpers import rel_err
    job = W.sk_ok_256x256x64(shape=(36, 30, 12), seed=43)
    job["values"] = (job["values"] - np.where(job["mask"] > 0, 0.4, 0.0)).astype(np.float32)
    p = job["params"][0]
    cm = geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], angles=p["angles"], sill=p["sill"],
                             nugget=p["nugget"])
    out = geo.simple_kriging(_cont_prop(job), geo.SugarboxGrid(36, 30, 12), p["radii"], p["max_neighbours"], cm,
                             mean=None, precision=precision)
    ref = O.run(job, kind="sk", sk_auto_mean=True, dumps=False)
    data = out.data.reshape(-1, order="F")
    assert np.array_equal(out.mask.reshape(-1, order="F"), ref["out_mask"])
    if precision == "fp64":
        assert np.array_equal(data.view(np.uint32), ref["out"].view(np.uint32))
    else:
        scale = float(np.max(np.abs(job["values"][job["mask"] > 0])))
        assert rel_err(data, ref["out"], 1e-6 * scale).max() <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_lvm_kriging_entry(native_lib, precision):
    """geo.lvm_kriging -> hpgl_lvm_kriging (api.cpp:344-383) with a mean cube,
    Gaussian variogram and clustered data (singular systems included)."""
    from hpgl_b200.geo_bsd import geo
    from tests.helpers import rel_err
    job = W.lvm_512x512x32(shape=(64, 64, 12), seed=44, blobs=20)
    p = job["params"][0]
    cm = geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], angles=p["angles"], sill=p["sill"],
                             nugget=p["nugget"])
    out = geo.lvm_kriging(_cont_prop(job), geo.SugarboxGrid(64, 64, 12), job["mean"], p["radii"],
                          p["max_neighbours"], cm, precision=precision)
    ref = O.run(job, kind="lvm", dumps=False)
    data = out.data.reshape(-1, order="F")
    assert np.array_equal(out.mask.reshape(-1, order="F"), ref["out_mask"])
    if precision == "fp64":
        assert np.array_equal(data.view(np.uint32), ref["out"].view(np.uint32))
    else:
        scale = float(np.max(np.abs(job["values"][job["mask"] > 0])))
        assert rel_err(data, ref["out"], 1e-6 * scale).max() <= 1e-6
