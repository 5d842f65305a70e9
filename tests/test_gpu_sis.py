"""Sequential indicator simulation on the GPU against the CPU restatement,
code for code: several categories with their own variograms and neighbour
counts, median SIS (two categories), the mean-cube form with and without
correlogram weights, a simulation mask, a category of more than 32
neighbours, and the reference's C entry points."""

import ctypes as C

import numpy as np
import pytest

from hpgl_b200 import native as N
from oracle import oracle as O
from sis_cases import case, means, params

pytestmark = pytest.mark.gpu


def _job(c, ps):
    return dict(c, params=ps)


@pytest.mark.parametrize("K", [2, 3, 4])
def test_sis_matches_oracle(native_lib, K):
    c = case(shape=(26, 22, 8), K=K, seed=K)
    ps = params(K)
    r = N.simulate_indicator(_job(c, ps), 1234)
    codes, mask = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=1234)
    assert np.array_equal(r["out"], codes) and np.array_equal(r["out_mask"], mask)


@pytest.mark.parametrize("correlogram", [False, True])
def test_sis_lvm_matches_oracle(native_lib, correlogram):
    c = case(shape=(22, 20, 8), K=3, seed=11)
    ps = [dict(p, marginal_prob=0.0) for p in params(3)]
    lv = means(c["shape"], 3)
    r = N.simulate_indicator(_job(c, ps), 77, category_means=lv, correlogram=correlogram)
    codes, mask = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=77, lvm=lv, correlogram=correlogram)
    assert np.array_equal(r["out"], codes) and np.array_equal(r["out_mask"], mask)


@pytest.mark.parametrize("correlogram", [False, True])
def test_sis_mask_and_64_neighbours(native_lib, correlogram):
    c = case(shape=(24, 20, 10), K=3, seed=12)
    ps = params(3, big=True)
    sm = (np.random.default_rng(4).random(c["codes"].size) < 0.6).astype(np.uint8)
    lv = means(c["shape"], 3, seed=13) if correlogram else None
    r = N.simulate_indicator(_job(c, ps), 31, simulation_mask=sm, category_means=lv, correlogram=correlogram)
    codes, mask = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=31, sim_mask=sm, lvm=lv,
                        correlogram=correlogram)
    assert np.array_equal(r["out"], codes) and np.array_equal(r["out_mask"], mask)


@pytest.mark.parametrize("nmax", [24, 32])
def test_sis_17_to_32_neighbours(native_lib, nmax):
    # the largest category decides the kernel: 17-32 neighbours take the
    # 32-column systems
    c = case(shape=(22, 20, 8), K=3, seed=19)
    ps = params(3)
    ps[2] = dict(ps[2], max_neighbours=nmax)
    r = N.simulate_indicator(_job(c, ps), 2468)
    codes, mask = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=2468)
    assert np.array_equal(r["out"], codes) and np.array_equal(r["out_mask"], mask)


def test_sis_reference_entry_points(native_lib):
    c = case(shape=(20, 18, 6), K=3, seed=14)
    ps = params(3)
    sh = O._shape(c["shape"])
    codes = c["codes"].copy()
    mask = c["mask"].copy()
    arr = O.HpglIndMaskedArray(codes.ctypes.data_as(C.POINTER(C.c_ubyte)), mask.ctypes.data_as(C.POINTER(C.c_ubyte)),
                               sh, 3)
    native_lib.hpgl_sis_simulation(C.byref(arr), O.ik_params_array(ps), 3, 4321, None)
    assert native_lib.hpgl_get_last_error() == 0
    want = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=4321)
    assert np.array_equal(codes, want[0]) and np.array_equal(mask, want[1])
    # the mean-cube form through hpgl_sis_simulation_lvm
    lv = means(c["shape"], 3, seed=15)
    codes = c["codes"].copy()
    mask = c["mask"].copy()
    arr = O.HpglIndMaskedArray(codes.ctypes.data_as(C.POINTER(C.c_ubyte)), mask.ctypes.data_as(C.POINTER(C.c_ubyte)),
                               sh, 3)
    fa = (O.HpglFloatArray * 3)(*[O.HpglFloatArray(a.ctypes.data_as(C.POINTER(C.c_float)), sh) for a in lv])
    native_lib.hpgl_sis_simulation_lvm(C.byref(arr), O.ik_params_array(ps), fa, 3, 4321, None, 1)
    assert native_lib.hpgl_get_last_error() == 0
    want = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=4321, lvm=lv, correlogram=True)
    assert np.array_equal(codes, want[0]) and np.array_equal(mask, want[1])


def test_sis_window_does_not_change_results(native_lib):
    c = case(shape=(120, 100, 24), K=4, seed=16, informed=0.01)
    ps = params(4)
    runs = []
    try:
        for window in (0, 300):
            native_lib.hpgl_b200_set_sim_window(window)
            runs.append(N.simulate_indicator(_job(c, ps), 3241347))
    finally:
        native_lib.hpgl_b200_set_sim_window(0)
    assert np.array_equal(runs[0]["out"], runs[1]["out"]) and runs[0]["out_mask"].all()


@pytest.mark.parametrize("lvm", [False, True])
def test_geo_bsd_sis_simulation(native_lib, lvm):
    from hpgl_b200.geo_bsd import geo, sis
    c = case(shape=(20, 16, 8), K=3, seed=17)
    ps = params(3)
    nx, ny, nz = c["shape"]
    f = lambda a: np.asfortranarray(np.reshape(a, c["shape"], order="F"))
    prop = (f(c["codes"]), f(c["mask"]), 3)
    data = [{"cov_model": geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], angles=p["angles"],
                                               sill=p["sill"], nugget=p["nugget"]),
             "radiuses": p["radii"], "max_neighbours": p["max_neighbours"]} for p in ps]
    if lvm:
        lv = means(c["shape"], 3, seed=18)
        out = sis.sis_simulation(prop, geo.SugarboxGrid(nx, ny, nz), data, 555, [f(a) for a in lv])
        want = O.sis(c["shape"], c["codes"], c["mask"], [dict(p, marginal_prob=0.0) for p in ps], seed=555, lvm=lv,
                     correlogram=True)
    else:
        out = sis.sis_simulation(prop, geo.SugarboxGrid(nx, ny, nz), data, 555, [p["marginal_prob"] for p in ps])
        want = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=555)
    assert np.array_equal(out.data.ravel(order="F"), want[0]) and np.array_equal(out.mask.ravel(order="F"), want[1])


@pytest.mark.parametrize("path", __import__("sim_golden").paths("sis"), ids=lambda p: p.split("/")[-1])
def test_gpu_matches_golden(native_lib, path):
    import sim_golden as SG
    d = SG.load(path)
    job = dict(shape=d["shape"], codes=d["codes"], mask=d["mask"], values=None, kind="ik", params=d["params"])
    r = N.simulate_indicator(job, d["seed"], category_means=list(d["lvm"]) if "lvm" in d else None,
                             correlogram=bool(d["correlogram"]))
    assert np.array_equal(r["out"], d["out_codes"]) and np.array_equal(r["out_mask"], d["out_mask"])
