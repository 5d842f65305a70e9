"""Sequential Gaussian simulation on the GPU against the CPU restatement:
every simulated value bit for bit (the speculative rounds reproduce the
sequential order exactly), for SK (mean 0), OK and LVM, with a simulation
mask, with up to 16, 32 and 64 neighbours, with CDF transforms, through the
reference's C entry points and the geo_bsd wrapper, and independent of the
rounds' window."""

import ctypes as C

import numpy as np
import pytest

from hpgl_b200 import native as N
from hpgl_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _job(shape, seed, n=12, cov=W.SPHERICAL, radii=None, informed=None):
    j = W.ok_50x50x20(shape=shape, seed=seed)
    p = dict(j["params"][0], max_neighbours=n, cov_type=cov)
    if radii:
        p["radii"] = radii
    j["params"] = [p]
    return j


def _same(a, b):
    # bit for bit, except that a NaN matches a NaN: where a negative kriging
    # variance meets the square root, the reference's x86 arithmetic gives its
    # default NaN (sign set) and the GPU its canonical NaN, and later nodes
    # that krige from such a node carry the NaN on
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32))


@pytest.mark.parametrize("kind", ["sk", "ok"])
@pytest.mark.parametrize("seed", [1, 31337])
def test_sgs_matches_oracle(native_lib, kind, seed):
    job = _job((24, 20, 8), seed=5)
    r = N.simulate(job, seed, kind=kind)
    v, m, _ = O.sgs(job, ordinary=kind == "ok", seed=seed)
    assert _same(r["out"], v) and np.array_equal(r["out_mask"], m)


def test_sgs_lvm_mask_64_neighbours(native_lib):
    job = _job((20, 18, 10), seed=6, n=40, cov=W.EXPONENTIAL, radii=(12, 12, 6))
    rng = np.random.default_rng(8)
    job["kind"] = "lvm"
    job["mean"] = (0.2 * rng.normal(size=job["values"].size)).astype(np.float32)
    sm = (rng.random(job["values"].size) < 0.7).astype(np.uint8)
    r = N.simulate(job, 77, kind="lvm", simulation_mask=sm)
    v, m, _ = O.sgs(job, seed=77, sim_mask=sm, lvm=job["mean"])
    assert _same(r["out"], v) and np.array_equal(r["out_mask"], m)


def test_sgs_ordinary_64_neighbours(native_lib):
    job = _job((18, 16, 10), seed=21, n=44, cov=W.GAUSSIAN, radii=(9, 9, 5))
    r = N.simulate(job, 4040, kind="ok")
    v, m, _ = O.sgs(job, ordinary=True, seed=4040)
    assert _same(r["out"], v) and np.array_equal(r["out_mask"], m)


def test_sgs_larger_grid(native_lib):
    job = _job((64, 60, 16), seed=7, n=24, radii=(10, 10, 4))
    r = N.simulate(job, 2024, kind="sk")
    v, m, _ = O.sgs(job, seed=2024)
    assert _same(r["out"], v) and np.array_equal(r["out_mask"], m)


def test_sgs_reference_entry_point(native_lib):
    job = _job((18, 16, 6), seed=8)
    nx, ny, nz = job["shape"]
    values = np.array(job["values"], np.float32)
    mask = np.array(job["mask"], np.uint8)
    arr = O.HpglContArray(values.ctypes.data_as(C.POINTER(C.c_float)), mask.ctypes.data_as(C.POINTER(C.c_ubyte)),
                          O._shape((nx, ny, nz)))
    p = job["params"][0]
    q = O.HpglSgsParams()
    q.covariance_type = p["cov_type"]
    q.ranges[:] = p["ranges"]
    q.angles[:] = p["angles"]
    q.sill, q.nugget = p["sill"], p["nugget"]
    q.radiuses[:] = p["radii"]
    q.max_neighbours = p["max_neighbours"]
    q.kriging_kind = 0  # ordinary
    q.seed = 555
    native_lib.hpgl_sgs_simulation(C.byref(arr), C.byref(q), None, None, None)
    assert native_lib.hpgl_get_last_error() == 0
    v, m, _ = O.sgs(job, ordinary=True, seed=555)
    assert _same(values, v) and np.array_equal(mask, m)


def _calc_cdf(values, mask):
    v = np.asarray(values, np.float32)[np.asarray(mask) != 0]
    u, c = np.unique(v, return_counts=True)
    size = u.size - 1 if u.size > 1 else u.size
    return u[:size], np.cumsum(c[:size] / float(v.size)).astype(np.float32)


def _geo(job):
    from hpgl_b200.geo_bsd import geo
    nx, ny, nz = job["shape"]
    p = job["params"][0]
    cov = geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], angles=p["angles"], sill=p["sill"],
                              nugget=p["nugget"])
    prop = geo.ContProperty(np.asfortranarray(np.reshape(job["values"], (nx, ny, nz), order="F")),
                            np.asfortranarray(np.reshape(job["mask"], (nx, ny, nz), order="F")))
    return geo, geo.SugarboxGrid(nx, ny, nz), prop, cov


@pytest.mark.parametrize("kriging_type", ["sk", "ok"])
def test_sgs_simulation_with_cdf(native_lib, kriging_type):
    from hpgl_b200.geo_bsd import sgs
    from hpgl_b200.geo_bsd.cdf import calc_cdf
    job = _job((22, 20, 8), seed=13)
    geo, grid, prop, cov = _geo(job)
    cdf = calc_cdf(prop)
    out = sgs.sgs_simulation(prop, grid, cdf, job["params"][0]["radii"], 12, cov, 4242, kriging_type=kriging_type)
    # the wrapper normalises the covariance to sill - nugget = 1 (sill 1, nugget 0 here: unchanged)
    v, m, _ = O.sgs(job, ordinary=kriging_type == "ok", seed=4242, cdf=(cdf.values, cdf.probs))
    assert _same(out.data.ravel(order="F"), v) and np.array_equal(out.mask.ravel(order="F"), m)


def test_sgs_simulation_lvm_cdf_and_mask(native_lib):
    from hpgl_b200.geo_bsd import sgs
    job = _job((20, 16, 8), seed=14, n=20, radii=(10, 10, 5))
    geo, grid, prop, cov = _geo(job)
    rng = np.random.default_rng(21)
    mean = np.asfortranarray((0.3 * rng.normal(size=prop.data.shape)).astype(np.float32))
    sm = np.asfortranarray((rng.random(prop.data.shape) < 0.5).astype(np.uint8))
    cdf = _calc_cdf(job["values"], job["mask"])
    out = sgs.sgs_simulation((prop.data, prop.mask), grid, (prop.data, prop.mask), (10, 10, 5), 20, cov, 99,
                             mean=mean, mask=sm)
    v, m, _ = O.sgs(job, seed=99, lvm=mean.ravel(order="F"), sim_mask=sm.ravel(order="F"), cdf=cdf)
    assert _same(out.data.ravel(order="F"), v) and np.array_equal(out.mask.ravel(order="F"), m)


def test_unconditional_simulation(native_lib):
    from hpgl_b200.geo_bsd import sgs
    job = _job((24, 22, 6), seed=15, radii=(8, 8, 4))
    geo, grid, prop, cov = _geo(job)
    out = sgs.sgs_simulation(prop, grid, None, (8, 8, 4), 12, cov, 7, use_harddata=False)
    empty = dict(job, values=np.zeros_like(job["values"]), mask=np.zeros_like(job["mask"]))
    v, m, _ = O.sgs(empty, seed=7)
    assert _same(out.data.ravel(order="F"), v) and np.array_equal(out.mask.ravel(order="F"), m)


def test_window_bounds_do_not_change_results(native_lib):
    # 166 x 141 x 40 cube, 1 % informed, radii 20, 12 neighbours: the result
    # is the sequential one whatever the speculative window, and the rounds
    # are few compared with the nodes
    job = _job((166, 141, 40), seed=16, n=12, cov=W.EXPONENTIAL, radii=(20, 20, 20))
    rng = np.random.default_rng(2)
    job["mask"] = (rng.random(job["values"].size) < 0.01).astype(np.uint8)
    runs = []
    try:
        for window in (0, 512, 1 << 20):
            native_lib.hpgl_b200_set_sim_window(window)
            assert native_lib.hpgl_get_last_error() == 0
            r = N.simulate(job, 3439275, kind="sk")
            runs.append(r)
    finally:
        native_lib.hpgl_b200_set_sim_window(0)
    for r in runs[1:]:
        assert _same(r["out"], runs[0]["out"]) and np.array_equal(r["out_mask"], runs[0]["out_mask"])
    assert runs[0]["rounds"] < 1000
    assert int(runs[0]["out_mask"].sum()) == job["values"].size


@pytest.mark.parametrize("path", __import__("sim_golden").paths("sgs"), ids=lambda p: p.split("/")[-1])
def test_gpu_matches_golden(native_lib, path):
    # through the reference's C entry points (the CDF transforms included)
    import sim_golden as SG
    d = SG.load(path)
    kw = SG.sgs_kwargs(d)
    values = np.array(d["values"], np.float32)
    mask = np.array(d["mask"], np.uint8)
    sh = O._shape(d["shape"])
    arr = O.HpglContArray(values.ctypes.data_as(C.POINTER(C.c_float)), mask.ctypes.data_as(C.POINTER(C.c_ubyte)), sh)
    p = d["params"][0]
    q = O.HpglSgsParams()
    q.covariance_type = p["cov_type"]
    q.ranges[:] = p["ranges"]
    q.angles[:] = p["angles"]
    q.sill, q.nugget = p["sill"], p["nugget"]
    q.radiuses[:] = p["radii"]
    q.max_neighbours = p["max_neighbours"]
    q.kriging_kind = 0 if kw["ordinary"] else 1
    q.seed = kw["seed"]
    keep = []
    cdfp = smp = None
    if "cdf" in kw:
        cv, cp = (np.ascontiguousarray(a, np.float32) for a in kw["cdf"])
        keep += [cv, cp]
        cdfp = C.byref(O.HpglNonParametricCdf(cv.ctypes.data_as(C.POINTER(C.c_float)),
                                              cp.ctypes.data_as(C.POINTER(C.c_float)), cv.size))
    if "sim_mask" in kw:
        sm = np.ascontiguousarray(kw["sim_mask"], np.uint8)
        keep.append(sm)
        smp = C.byref(O.HpglUbyteArray(sm.ctypes.data_as(C.POINTER(C.c_ubyte)), sh))
    if "lvm" in kw:
        lv = np.ascontiguousarray(kw["lvm"], np.float32)
        keep.append(lv)
        fa = O.HpglFloatArray(lv.ctypes.data_as(C.POINTER(C.c_float)), sh)
        native_lib.hpgl_sgs_lvm_simulation(C.byref(arr), C.byref(q), cdfp, C.byref(fa), smp)
    else:
        native_lib.hpgl_sgs_simulation(C.byref(arr), C.byref(q), cdfp, None, smp)
    assert native_lib.hpgl_get_last_error() == 0
    assert _same(values, d["out_values"]) and np.array_equal(mask, d["out_mask"])


def test_sgs_refuses_negative_seed_without_touching_data(native_lib):
    # the reference's walk leaves the grid for a seed negative as an int; here
    # the call is refused before the CDF transform changes the property
    job = _job((12, 10, 4), seed=20)
    values = np.array(job["values"], np.float32)
    mask = np.array(job["mask"], np.uint8)
    before = values.copy()
    sh = O._shape(job["shape"])
    arr = O.HpglContArray(values.ctypes.data_as(C.POINTER(C.c_float)), mask.ctypes.data_as(C.POINTER(C.c_ubyte)), sh)
    p = job["params"][0]
    q = O.HpglSgsParams()
    q.covariance_type = p["cov_type"]
    q.ranges[:] = p["ranges"]
    q.angles[:] = p["angles"]
    q.sill, q.nugget = p["sill"], p["nugget"]
    q.radiuses[:] = p["radii"]
    q.max_neighbours = p["max_neighbours"]
    q.kriging_kind = 1
    cv = np.sort(values[mask != 0])[:-1].copy()
    cp = np.linspace(0.1, 0.9, cv.size).astype(np.float32)
    cdf = O.HpglNonParametricCdf(cv.ctypes.data_as(C.POINTER(C.c_float)), cp.ctypes.data_as(C.POINTER(C.c_float)),
                                 cv.size)
    for seed in (-1, 2 ** 31 + 7):
        q.seed = seed
        native_lib.hpgl_sgs_simulation(C.byref(arr), C.byref(q), C.byref(cdf), None, None)
        assert native_lib.hpgl_get_last_error() == N.HPGL_E_INVALID
        assert np.array_equal(values, before)
    # a seed above 2^32 is taken modulo 2^32, as the reference's int and uint32 casts do
    q.seed = 2 ** 32 + 9
    native_lib.hpgl_sgs_simulation(C.byref(arr), C.byref(q), None, None, None)
    assert native_lib.hpgl_get_last_error() == 0
    v, m, _ = O.sgs(job, seed=9)
    assert _same(values, v) and np.array_equal(mask, m)
