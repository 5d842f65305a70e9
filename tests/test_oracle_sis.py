"""The CPU restatement of sequential indicator simulation (oracle/hpgl_oracle.cpp:
do_sis with per-category simple kriging, median SIS for two categories, the
mean-cube form with and without correlogram weights, the draw from the
float probabilities) against the reference's own sources compiled by
oracle/build_ref.sh."""

import numpy as np
import pytest

from oracle import oracle as O
from sis_cases import case, means, params

need_ref = pytest.mark.skipif(not O.reference_available(), reason="compiled reference not present")


@need_ref
@pytest.mark.parametrize("K", [2, 3, 4])
@pytest.mark.parametrize("seed", [17, 99991])
def test_sis_matches_reference(K, seed):
    c = case(K=K, seed=K)
    ps = params(K)
    a = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=seed)
    b = O.ref_sis(c["shape"], c["codes"], c["mask"], ps, seed=seed)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@need_ref
@pytest.mark.parametrize("correlogram", [False, True])
def test_sis_lvm_matches_reference(correlogram):
    c = case(K=3, seed=8)
    ps = [dict(p, marginal_prob=0.0) for p in params(3)]
    lv = means(c["shape"], 3)
    a = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=23, lvm=lv, correlogram=correlogram)
    b = O.ref_sis(c["shape"], c["codes"], c["mask"], ps, seed=23, lvm=lv, correlogram=correlogram)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@need_ref
def test_sis_mask_and_many_neighbours_match_reference():
    c = case(shape=(20, 18, 8), K=3, seed=9)
    ps = params(3, big=True)
    sm = (np.random.default_rng(4).random(c["codes"].size) < 0.5).astype(np.uint8)
    a = O.sis(c["shape"], c["codes"], c["mask"], ps, seed=29, sim_mask=sm)
    b = O.ref_sis(c["shape"], c["codes"], c["mask"], ps, seed=29, sim_mask=sm)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_informed_codes_are_kept_and_every_node_simulated():
    c = case(shape=(24, 20, 6), K=3, seed=10, informed=0.05)
    codes, mask = O.sis(c["shape"], c["codes"], c["mask"], params(3), seed=5)
    inf = c["mask"] != 0
    assert mask.all() and np.array_equal(codes[inf], c["codes"][inf]) and codes.max() < 3


@pytest.mark.parametrize("path", __import__("sim_golden").paths("sis"), ids=lambda p: p.split("/")[-1])
def test_oracle_matches_golden(path):
    import sim_golden as SG
    d = SG.load(path)
    codes, mask = O.sis(d["shape"], d["codes"], d["mask"], d["params"], seed=d["seed"],
                        lvm=list(d["lvm"]) if "lvm" in d else None, correlogram=bool(d["correlogram"]))
    assert np.array_equal(codes, d["out_codes"]) and np.array_equal(mask, d["out_mask"])


@need_ref
@pytest.mark.parametrize("shape", [(2, 1, 1), (4, 1, 1), (3, 2, 1), (2, 2, 2), (3, 2, 2), (3, 3, 1)])
def test_tiny_grids_match_reference(shape):
    # including the sizes whose path repeats nodes (2, 4, 6, 8, 12)
    n = int(np.prod(shape))
    rng = np.random.default_rng(n)
    codes = rng.integers(0, 3, n).astype(np.uint8)
    mask = (rng.random(n) < 0.3).astype(np.uint8)
    ps = [dict(p, radii=(2, 2, 2), max_neighbours=4) for p in params(3)]
    for seed in (0, 3):
        a = O.sis(shape, codes, mask, ps, seed=seed)
        b = O.ref_sis(shape, codes, mask, ps, seed=seed)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
