"""The CPU restatement of the experimental variograms and layer stacking
(oracle/variogram_oracle.cpp) against the reference's _cvariogram sources
compiled by oracle/build_ref.sh, the reference's own test vectors
(_cvariogram/v_test.py) and the committed fixtures
(tests/golden/make_golden_variogram.py)."""

import ctypes as C
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
import variogram_cases as VC

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "variogram")
need_ref = pytest.mark.skipif(not O.reference_cv_available(), reason="compiled reference not present")


def _t(name):
    return O.cv_template(*VC.TEMPLATES[name])


def test_lag_areas_and_window_match_reference_test_vectors():
    # _cvariogram/v_test.py:44-67: ellipsoid (10, 20, 30) at (40, 50, 60),
    # lag width 10, separation 10, tolerance 0.5, 5 lags.  Its window values
    # come from directions built with numpy's pi; the library's directions
    # use 3.14159265358, so they agree to 1e-9 here.
    t = O.cv_template(10, 10, 0.5, 5, 0, (10, 20, 30), (40, 50, 60))
    lib = O.restated()
    lib.oracle_lag_areas.restype = C.c_longlong
    assert lib.oracle_lag_areas(C.byref(t)) == 76905
    w = (C.c_double * 6)()
    lib.oracle_template_window(C.byref(t), w)
    want = [-24.489718110804734, -28.156717480994359, -20.775222129826481, 49.109911936109938, 48.815513039321097,
            59.077444285775378]
    assert np.allclose(list(w), want, rtol=0, atol=1e-9)


@need_ref
def test_restated_geometry_matches_reference():
    ref = O.ref_cv()
    lib = O.restated()
    lib.oracle_lag_areas.restype = C.c_longlong
    for name, spec in VC.TEMPLATES.items():
        t = O.cv_template(*spec)
        e = O.CvEllipsoid()
        ref.fill_ellipsoid_directions(C.byref(e), C.c_double(spec[6][0]), C.c_double(spec[6][1]),
                                      C.c_double(spec[6][2]))
        for k in ("direction1", "direction2", "direction3"):
            assert list(getattr(e, k).data) == list(getattr(t.ellipsoid, k).data), name
        w1, w2 = (C.c_double * 6)(), (C.c_double * 6)()
        lib.oracle_template_window(C.byref(t), w1)
        ref.ref_cvar_window(C.byref(t), w2)
        assert list(w1) == list(w2), name
        assert lib.oracle_lag_areas(C.byref(t)) == ref.ref_cvar_lag_areas(C.byref(t)), name
        rng = np.random.default_rng(1)
        for v in rng.uniform(-30, 30, (500, 3)):
            assert lib.oracle_in_tunnel(C.byref(t), *map(C.c_double, v)) == \
                ref.ref_cvar_in_tunnel(C.byref(t), *map(C.c_double, v))


@need_ref
@pytest.mark.parametrize("name", list(VC.TEMPLATES))
@pytest.mark.parametrize("order", ["F", "C"])
def test_restated_grid_variograms_match_reference(name, order):
    t = _t(name)
    v, m = VC.grid((28, 22, 7), 0.3, seed=sum(map(ord, name)), order=order)
    o = O.variograms(t, v, m)
    r = O.ref_variograms(t, v, m)
    assert np.array_equal(o["result"].view(np.uint32), r.view(np.uint32))
    assert o["counts"].sum() > 0
    # the reference's sequential sums and the exact sums agree to rounding
    nz = o["counts"] > 0
    assert np.allclose(o["seq_sums"][nz], o["exact_sums"][nz], rtol=1e-12, atol=0)


@need_ref
def test_restated_grid_variograms_strided_view_and_extra_lags():
    t = _t("x_narrow")
    v, m = VC.grid((40, 30, 10), 0.2, seed=7)
    v2, m2 = v[::2, 1::2, :], m[::2, 1::2, :]  # a strided view of both
    o = O.variograms(t, v2, m2, lags=12)  # more result slots than lags
    r = O.ref_variograms(t, v2, m2, lags=12)
    assert np.array_equal(o["result"][:8].view(np.uint32), r[:8].view(np.uint32))


@need_ref
@pytest.mark.parametrize("name", list(VC.TEMPLATES))
def test_restated_point_variograms_match_reference(name):
    t = _t(name)
    xs, ys, zs, vals = VC.points(700, seed=3)
    o = O.variograms_points(t, xs, ys, zs, vals)
    r = O.ref_variograms_points(t, xs, ys, zs, vals)
    assert np.array_equal(o["result"].view(np.uint32), r.view(np.uint32))


@need_ref
def test_restated_stack_layers_match_reference():
    for seed in range(6):
        ls = VC.layers(17, 13, 7, seed)
        marks = list(range(1, 8))
        a = np.asfortranarray(np.full((17, 13, 12), -5, np.float32))
        b = a.copy(order="F")
        O.stack_layers(ls, marks, 12, 1.25, -1, a)
        O.stack_layers(ls, marks, 12, 1.25, -1, b, reference=True)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_oracle_matches_golden(path):
    g = np.load(path)
    spec = tuple(g["template"])
    t = O.cv_template(spec[0], spec[1], spec[2], int(spec[3]), spec[4], tuple(spec[5:8]), tuple(spec[8:11]))
    kind = str(g["kind"])
    if kind == "grid":
        o = O.variograms(t, g["values"], g["mask"])
    elif kind == "points":
        o = O.variograms_points(t, g["xs"], g["ys"], g["zs"], g["vals"])
    else:
        res = np.asfortranarray(np.full(g["result"].shape, -5, np.float32))
        O.stack_layers(list(g["layers"]), list(g["markers"]), int(g["nz"]), float(g["scalez"]), int(g["blank"]), res)
        assert np.array_equal(res, g["result"])
        return
    assert np.array_equal(o["result"].view(np.uint32), g["result"].view(np.uint32))
