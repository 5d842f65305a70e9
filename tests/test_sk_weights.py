"""hpgl_simple_kriging_weights (api.cpp:292-342): SK weights of one point
from explicit neighbour coordinates.

CPU: the oracle restatement equals the compiled reference bit for bit.
GPU: the library's entry point agrees with the oracle to 1e-6 relative (the
device evaluates exp/pow of continuous offsets with CUDA's libm, so a weight
may differ in its last float bits)."""

import numpy as np
import pytest

from hpgl_b200 import native as N
from hpgl_b200 import workloads as W
from oracle import oracle as O


def _cases(seed, count, nmax=60):
    rng = np.random.default_rng(seed)
    for _ in range(count):
        n = int(rng.integers(1, nmax))
        ct = int(rng.integers(0, 3))
        p = W.cov_params(ct, rng.uniform(5, 40, 3), angles=rng.uniform(0, 90, 3), sill=1.0,
                         nugget=rng.uniform(0.01, 0.2))
        pts = rng.uniform(0, 30, (n, 3)).astype(np.float32)
        c = rng.uniform(0, 30, 3).astype(np.float32)
        yield c, pts, p


@pytest.mark.skipif(not O.reference_available(), reason="reference library not built here")
def test_oracle_matches_reference():
    for c, pts, p in _cases(1, 200):
        rc, w = O.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p)
        if rc:
            continue
        wr = O.ref_sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p)
        assert np.array_equal(w.view(np.uint32), wr.view(np.uint32))


@pytest.mark.gpu
def test_gpu_matches_oracle(native_lib):
    checked = 0
    for c, pts, p in _cases(2, 120):
        rc, wo = O.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p)
        if rc:
            with pytest.raises(N.HpglError):
                N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p)
            continue
        wg = N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p)
        scale = max(1e-3, float(np.max(np.abs(wo))))
        assert np.max(np.abs(wg - wo)) <= 1e-6 * scale
        checked += 1
    assert checked > 50


@pytest.mark.gpu
def test_gpu_zero_and_errors(native_lib):
    p = W.cov_params(1, (10, 10, 10))
    w = N.sk_weights((0, 0, 0), [], [], [], p)
    assert w.size == 0
    bad = dict(p, ranges=(0.0, 10.0, 10.0))
    with pytest.raises(N.HpglError) as e:
        N.sk_weights((0, 0, 0), [1.0], [1.0], [1.0], bad)
    assert e.value.code == N.HPGL_E_INVALID
