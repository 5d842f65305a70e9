"""The CPU restatement of sequential Gaussian simulation (oracle/hpgl_oracle.cpp:
random path, boost::mt11213b draws, Odeh-Evans quantile, kriging from the
informed and already simulated nodes) against the reference's own sources
compiled by oracle/build_ref.sh, whose missing pieces are supplied as
oracle/ref_shim's boost::mt11213b and oracle/gen_primes.py's prime table."""

import numpy as np
import pytest

from hpgl_b200 import workloads as W
from oracle import oracle as O

need_ref = pytest.mark.skipif(not O.reference_available(), reason="compiled reference not present")


def _job(shape=(20, 18, 6), seed=4, n=12, cov=W.SPHERICAL):
    j = W.ok_50x50x20(shape=shape, seed=seed)
    j["params"] = [dict(j["params"][0], max_neighbours=n, cov_type=cov)]
    return j


@need_ref
@pytest.mark.parametrize("ordinary", [False, True])
@pytest.mark.parametrize("seed", [1, 7, 123456])
def test_sgs_matches_reference(ordinary, seed):
    job = _job()
    v1, m1, order = O.sgs(job, ordinary=ordinary, seed=seed)
    v2, m2 = O.ref_sgs(job, ordinary=ordinary, seed=seed)
    assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32))
    assert np.array_equal(m1, m2)
    assert len(order) == int((job["mask"] == 0).sum())


@need_ref
def test_sgs_lvm_mask_and_exponential_match_reference():
    job = _job(shape=(16, 14, 8), seed=9, n=20, cov=W.EXPONENTIAL)
    rng = np.random.default_rng(3)
    lvm = (0.1 * rng.normal(size=job["values"].size)).astype(np.float32)
    sm = (rng.random(job["values"].size) < 0.6).astype(np.uint8)
    v1, m1, _ = O.sgs(job, seed=5, sim_mask=sm, lvm=lvm)
    v2, m2 = O.ref_sgs(job, seed=5, sim_mask=sm, lvm=lvm)
    assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32)) and np.array_equal(m1, m2)


def test_path_visits_every_node_once():
    # the walk is a full-period LCG: the simulation order is a permutation of
    # the uninformed nodes
    job = _job(shape=(17, 11, 5), seed=2)
    _, _, order = O.sgs(job, seed=99)
    uninformed = np.nonzero(job["mask"] == 0)[0]
    assert sorted(order.tolist()) == uninformed.tolist()


def test_draws_are_standard_normal():
    xp = O.sgs_draws(42, 200000)
    assert abs(xp.mean()) < 0.01 and abs(xp.std() - 1) < 0.01


def _calc_cdf(values, mask):
    v = np.asarray(values, np.float32)[np.asarray(mask) != 0]
    u, c = np.unique(v, return_counts=True)
    size = u.size - 1 if u.size > 1 else u.size
    return u[:size], np.cumsum(c[:size] / float(v.size)).astype(np.float32)


@need_ref
@pytest.mark.parametrize("ordinary", [False, True])
def test_sgs_cdf_transform_matches_reference(ordinary):
    job = _job(seed=11)
    cdf = _calc_cdf(job["values"], job["mask"])
    v1, m1, _ = O.sgs(job, ordinary=ordinary, seed=3, cdf=cdf)
    v2, m2 = O.ref_sgs(job, ordinary=ordinary, seed=3, cdf=cdf)
    assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32)) and np.array_equal(m1, m2)


@need_ref
def test_sgs_lvm_cdf_matches_reference():
    job = _job(shape=(16, 14, 8), seed=12)
    rng = np.random.default_rng(5)
    lvm = (0.1 * rng.normal(size=job["values"].size)).astype(np.float32)
    cdf = _calc_cdf(job["values"], job["mask"])
    v1, m1, _ = O.sgs(job, seed=8, lvm=lvm, cdf=cdf)
    v2, m2 = O.ref_sgs(job, seed=8, lvm=lvm, cdf=cdf)
    assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32)) and np.array_equal(m1, m2)


def test_cdf_transform_round_trip_is_close():
    # the back transform undoes the forward one up to the interpolation's
    # float rounding (a property of the restated transforms, not of the data)
    rng = np.random.default_rng(1)
    vals = np.sort(rng.normal(size=200).astype(np.float32))
    cdf = (vals[:-1], np.cumsum(np.full(199, 1 / 200.0)).astype(np.float32))
    x = vals[10:150]
    g = O.cdf_transform(x, cdf, 0)
    back = O.cdf_transform(g, cdf, 1)
    assert np.allclose(back, x, atol=2e-3)


@pytest.mark.parametrize("path", __import__("sim_golden").paths("sgs"), ids=lambda p: p.split("/")[-1])
def test_oracle_matches_golden(path):
    import sim_golden as SG
    d = SG.load(path)
    job = dict(shape=d["shape"], values=d["values"], mask=d["mask"], params=d["params"])
    v, m, _ = O.sgs(job, **SG.sgs_kwargs(d))
    assert np.array_equal(v.view(np.uint32), d["out_values"].view(np.uint32)) and np.array_equal(m, d["out_mask"])


@need_ref
@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 1, 1), (4, 1, 1), (3, 2, 1), (2, 2, 2), (3, 2, 2), (5, 1, 1),
                                   (3, 3, 1)])
def test_tiny_grids_match_reference(shape):
    # grids whose path repeats nodes (sizes 2, 4, 6, 8, 12) and other tiny ones
    rng = np.random.default_rng(sum(shape))
    n = int(np.prod(shape))
    job = dict(shape=shape, values=rng.normal(size=n).astype(np.float32),
               mask=(rng.random(n) < 0.3).astype(np.uint8),
               params=[dict(cov_type=0, ranges=(3.0, 3.0, 3.0), angles=(0.0, 0.0, 0.0), sill=1.0, nugget=0.0,
                            radii=(2, 2, 2), max_neighbours=4)])
    for seed in (0, 1, 5):
        v1, m1, _ = O.sgs(job, seed=seed)
        v2, m2 = O.ref_sgs(job, seed=seed)
        assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32)) and np.array_equal(m1, m2)


@need_ref
def test_simulation_mask_values_other_than_one_are_skipped():
    # the reference simulates a node only where the simulation mask is exactly 1
    job = _job(shape=(14, 12, 4), seed=13)
    rng = np.random.default_rng(6)
    sm = rng.integers(0, 3, job["values"].size).astype(np.uint8)
    v1, m1, _ = O.sgs(job, seed=21, sim_mask=sm)
    v2, m2 = O.ref_sgs(job, seed=21, sim_mask=sm)
    assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32)) and np.array_equal(m1, m2)
    assert not m1[(sm == 2) & (job["mask"] == 0)].any()
