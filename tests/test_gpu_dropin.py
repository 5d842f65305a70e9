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
