"""Continuous batching (hpgl_b200_server_*): a stream of mixed OK/SK/IK jobs
of different grids and variograms, submitted faster than they complete so
they overlap on the GPU, gives for every job exactly the result of running
it alone; admission respects the HBM budget."""

import numpy as np
import pytest

from hpgl_b200 import native as N
from hpgl_b200 import serve as S
from hpgl_b200 import workloads as W


def _same(a, b):
    if a["out"].dtype == np.float32:
        assert np.array_equal(a["out"].view(np.uint32), b["out"].view(np.uint32))
    else:
        assert np.array_equal(a["out"], b["out"])
    assert np.array_equal(a["out_mask"], b["out_mask"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_results_alone_equal_results_in_the_mix(native_lib, precision):
    stream = W.serve_stream(24, rate_per_s=1e6, seed=31, max_cells=64 * 64 * 16)
    kinds = set(job["kind"] for _, job in stream)
    assert {"ok", "sk", "ik"} <= kinds
    with S.Server(hbm_budget_bytes=8 << 30, max_inflight=6) as srv:
        tickets = [srv.submit(job, precision=precision) for _, job in stream]
        mixed = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == 24 and st["failed"] == 0
    assert st["peak_inflight"] > 1, "jobs must overlap on the device"
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    for (_, job), got in zip(stream, mixed):
        alone = N.krige(job, precision=precision)
        _same(got, alone)


@pytest.mark.gpu
def test_admission_by_budget(native_lib):
    stream = W.serve_stream(6, rate_per_s=1e6, seed=32, max_cells=48 * 48 * 16)
    job0 = stream[0][1]
    with S.Server(hbm_budget_bytes=1 << 40, max_inflight=1) as srv:
        srv.result(srv.submit(job0))
    # a budget of one job at a time serialises the stream
    sizes = []
    for _, job in stream:
        with S.Server(hbm_budget_bytes=1 << 40, max_inflight=1) as srv:
            srv.result(srv.submit(job))
            sizes.append(srv.stats()["peak_bytes"])
    budget = max(sizes) + min(sizes) - 1  # never two of the largest at once
    with S.Server(hbm_budget_bytes=budget, max_inflight=6) as srv:
        ts = [srv.submit(job) for _, job in stream]
        for t in ts:
            srv.result(t)
        st = srv.stats()
    assert st["peak_bytes"] <= budget
    # a job larger than the whole budget fails with HPGL_E_CAPACITY
    with S.Server(hbm_budget_bytes=1 << 20, max_inflight=2) as srv:
        t = srv.submit(job0)
        assert srv.wait(t) == N.HPGL_E_CAPACITY
