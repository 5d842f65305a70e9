"""Experimental variograms and layer stacking on the GPU against the CPU
restatement (oracle/variogram_oracle.cpp) and the reference's results:
per-lag pair counts bit for bit, per-lag sums equal to the exact sums the
restatement accumulates, semivariances equal to the float of the exact
sum / count / 2 and within one float ulp of the reference's (whose
sequential double sums differ from the exact ones in their last bits), and
stacked cubes bit for bit."""

import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
import variogram_cases as VC

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "variogram")


@pytest.fixture(scope="module")
def CV():
    from hpgl_b200 import cvariogram
    return cvariogram


def gpu_template(CV, spec):
    ell = CV.Ellipsoid(spec[5][0], spec[5][1], spec[5][2], spec[6][0], spec[6][1], spec[6][2])
    return CV.VariogramSearchTemplate(spec[0], spec[1], spec[2], spec[3], spec[4], ell)


def expected_floats(exact_sums, counts):
    with np.errstate(divide="ignore", invalid="ignore"):
        return (exact_sums / counts.astype(np.float64) / 2).astype(np.float32)


def ulps(a, b):
    a = a.view(np.int32).astype(np.int64)
    b = b.view(np.int32).astype(np.int64)
    return np.abs(a - b)


@pytest.mark.parametrize("name", list(VC.TEMPLATES))
@pytest.mark.parametrize("order", ["F", "C"])
def test_grid_matches_oracle(CV, name, order):
    spec = VC.TEMPLATES[name]
    v, m = VC.grid((36, 29, 9), 0.3, seed=sum(map(ord, name)) + 1, order=order)
    o = O.variograms(O.cv_template(*spec), v, m)
    t = gpu_template(CV, spec)
    sums, counts = CV.CalcVariogramStats(t, hard_data=(v, m))
    assert np.array_equal(counts, o["counts"])
    assert np.array_equal(sums, o["exact_sums"])
    _, res = CV.CalcVariograms(t, (v, m))
    assert np.array_equal(res.view(np.uint32), expected_floats(o["exact_sums"], o["counts"]).view(np.uint32))
    ok = o["counts"] > 0
    assert ulps(res[ok], o["result"][ok]).max() <= 1
    assert np.all(np.isnan(res[~ok]))


def test_grid_strided_and_sampled(CV):
    spec = VC.TEMPLATES["overlapping_lags"]
    v, m = VC.grid((50, 40, 12), 0.25, seed=9)
    v2, m2 = v[1::2, ::3, :], m[1::2, ::3, :]
    t = gpu_template(CV, spec)
    ot = O.cv_template(*spec)
    o = O.variograms(ot, v2, m2)
    sums, counts = CV.CalcVariogramStats(t, hard_data=(v2, m2))
    assert np.array_equal(counts, o["counts"]) and np.array_equal(sums, o["exact_sums"])
    for pct in (0, 37, 100):
        o = O.variograms(ot, v, m, percent=pct)
        sums, counts = CV.CalcVariogramStats(t, hard_data=(v, m), percent=pct)
        assert np.array_equal(counts, o["counts"]) and np.array_equal(sums, o["exact_sums"]), pct


def test_grid_full_cube(CV):
    """166 x 141 x 20, 10 % informed: thousands of blocks per offset slice."""
    spec = VC.TEMPLATES["x_narrow"]
    v, m = VC.grid((166, 141, 20), 0.10, seed=11)
    o = O.variograms(O.cv_template(*spec), v, m)
    sums, counts = CV.CalcVariogramStats(gpu_template(CV, spec), hard_data=(v, m))
    assert np.array_equal(counts, o["counts"])
    assert np.array_equal(sums, o["exact_sums"])


@pytest.mark.parametrize("name", list(VC.TEMPLATES))
def test_points_match_oracle(CV, name):
    spec = VC.TEMPLATES[name]
    xs, ys, zs, vals = VC.points(1500, seed=sum(map(ord, name)))
    o = O.variograms_points(O.cv_template(*spec), xs, ys, zs, vals)
    t = gpu_template(CV, spec)
    ps = {"X": xs, "Y": ys, "Z": zs, "Property": vals}
    sums, counts = CV.CalcVariogramStats(t, point_set=ps)
    assert np.array_equal(counts, o["counts"])
    assert np.array_equal(sums, o["exact_sums"])
    _, res = CV.CalcVariogramsFromPointSet(t, ps)
    exp = expected_floats(o["exact_sums"], o["counts"])
    exp[o["counts"] == 0] = 0
    assert np.array_equal(res.view(np.uint32), exp.view(np.uint32))
    assert ulps(res, o["result"]).max() <= 1


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_golden(CV, path):
    g = np.load(path)
    s = tuple(g["template"])
    spec = (s[0], s[1], s[2], int(s[3]), s[4], tuple(s[5:8]), tuple(s[8:11]))
    kind = str(g["kind"])
    if kind == "stack":
        res = np.asfortranarray(np.full(g["result"].shape, -5, np.float32))
        CV.CStackLayers([np.asfortranarray(l) for l in g["layers"]], [int(x) for x in g["markers"]], int(g["nz"]),
                        float(g["scalez"]), int(g["blank"]), res)
        assert np.array_equal(res, g["result"])
        return
    t = gpu_template(CV, spec)
    if kind == "grid":
        _, res = CV.CalcVariograms(t, (g["values"], g["mask"]))
    else:
        _, res = CV.CalcVariogramsFromPointSet(t, {"X": g["xs"], "Y": g["ys"], "Z": g["zs"], "Property": g["vals"]})
    ok = ~np.isnan(g["result"])
    assert np.array_equal(np.isnan(res), ~ok)
    assert ulps(res[ok], g["result"][ok]).max() <= 1


def test_stack_layers(CV):
    for seed in range(4):
        ls = VC.layers(33, 27, 9, seed + 100)
        a = np.asfortranarray(np.full((33, 27, 16), -5, np.float32))
        b = a.copy(order="F")
        CV.CStackLayers(ls, list(range(1, 10)), 16, 1.3, -1, a)
        O.stack_layers(ls, list(range(1, 10)), 16, 1.3, -1, b)
        assert np.array_equal(a, b)
