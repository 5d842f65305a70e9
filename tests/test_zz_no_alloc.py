"""hpgl_b200_simple_kriging_weights_static: the simple-kriging-weights entry
point for callers that cannot allocate device memory (cudaMalloc/cudaFree
synchronise the device and stall the caller's other GPU work, and a host
that reserved the GPU's memory for its own pool leaves nothing to allocate).
It must give the same weights as hpgl_simple_kriging_weights, which
allocates its scratch -- bit for bit, the two run the same kernel on the same
inputs -- on consecutive calls that reuse its fixed scratch array, reject
neighbour counts above its stated maximum, and leave the device's free memory
unchanged (no allocation).

This file is named to be collected last."""

import numpy as np
import pytest

from hpgl_b200 import native as N
from hpgl_b200 import workloads as W

STATIC = "hpgl_b200_simple_kriging_weights_static"
ALLOC = "hpgl_simple_kriging_weights"
STATIC_MAX = 256   # HPGL_B200_STATIC_WEIGHTS_MAX in include/hpgl.h


def _case(rng, n):
    ct = int(rng.integers(0, 3))
    p = W.cov_params(ct, rng.uniform(5, 40, 3), angles=rng.uniform(0, 90, 3), sill=1.0,
                     nugget=rng.uniform(0.05, 0.2))
    pts = rng.uniform(0, 30, (n, 3)).astype(np.float32)
    c = rng.uniform(0, 30, 3).astype(np.float32)
    return c, pts, p


def _same(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.gpu
def test_static_entry_matches_allocating_entry(native_lib):
    rng = np.random.default_rng(11)
    compared = 0
    for n in (1, 7, 33, 64, 100, STATIC_MAX):
        c, pts, p = _case(rng, n)
        try:
            ref = N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p, entry=ALLOC)
        except N.HpglError:
            continue
        first = N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p, entry=STATIC)
        second = N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p, entry=STATIC)
        assert _same(first, ref), "first static call differs (n=%d)" % n
        assert _same(second, ref), "second static call differs (n=%d)" % n
        compared += 1
    assert compared >= 4


@pytest.mark.gpu
def test_static_entry_alternating_sizes(native_lib):
    # a large call leaves its contents in the shared scratch; the smaller
    # call after it must not see them
    rng = np.random.default_rng(12)
    big = _case(rng, 200)
    small = _case(rng, 9)
    for c, pts, p in (big, small, big, small):
        ref = N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p, entry=ALLOC)
        got = N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p, entry=STATIC)
        assert _same(got, ref)


@pytest.mark.gpu
def test_static_entry_rejects_above_maximum(native_lib):
    rng = np.random.default_rng(13)
    c, pts, p = _case(rng, STATIC_MAX + 1)
    with pytest.raises(N.HpglError) as e:
        N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p, entry=STATIC)
    assert e.value.code == N.HPGL_E_CAPACITY


@pytest.mark.gpu
def test_static_entry_does_not_allocate(native_lib):
    # the device's free memory is unchanged across static calls once the
    # first call has loaded the kernel (lazy module loading) and the context
    import torch
    rng = np.random.default_rng(14)
    c, pts, p = _case(rng, STATIC_MAX)
    N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p, entry=STATIC)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for n in (1, 64, STATIC_MAX, 5):
        c, pts, p = _case(rng, n)
        N.sk_weights(c, pts[:, 0], pts[:, 1], pts[:, 2], p, entry=STATIC)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
