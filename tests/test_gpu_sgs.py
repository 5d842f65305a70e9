"""Sequential Gaussian simulation on the GPU against the CPU restatement:
every simulated value bit for bit (the batches of mutually distant nodes
reproduce the sequential order exactly), for SK (mean 0), OK and LVM, with a
simulation mask, with more than 32 neighbours, and through the reference's
C entry points."""

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
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


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
