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


_stream_ref = {}


def _stream_with_oracle():
    """A seeded stream of the serving configuration (every kind with every
    variogram type, 13 to 64 neighbours, 33-40 k cells per job) and the
    oracle's results with per-node dumps."""
    from oracle import oracle as O
    if not _stream_ref:
        stream = W.serve_stream(16, rate_per_s=1e6, seed=42, max_cells=48 * 48 * 16)
        _stream_ref["stream"] = stream
        _stream_ref["ref"] = [O.run(job, dumps=True) for _, job in stream]
    return _stream_ref["stream"], _stream_ref["ref"]


def test_stream_covers_the_serving_mix():
    stream = W.serve_stream(16, rate_per_s=1e6, seed=42, max_cells=48 * 48 * 16)
    combos = set((job["kind"], job["params"][0]["cov_type"]) for _, job in stream)
    assert combos == {(k, c) for k in ("ok", "sk", "ik") for c in (0, 1, 2)}
    nmax = [job["params"][0]["max_neighbours"] for _, job in stream]
    assert max(nmax) == 64 and min(nmax) < 16 and sum(n > 32 for n in nmax) >= 5


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stream_jobs_match_the_oracle(native_lib, precision):
    """Every job of the stream, run in the mix, against the oracle: neighbour
    lists, statuses and masks bit-identical; FP64 estimates, weights and
    variances bit-identical; mixed estimates within 1e-6 relative (floor 1e-6
    of the field's scale), variances within 1e-6 relative (floor 1e-6 of the
    sill), IK categories identical."""
    from tests.helpers import rel_err
    stream, refs = _stream_with_oracle()
    with S.Server(hbm_budget_bytes=8 << 30, max_inflight=6) as srv:
        tickets = [srv.submit(job, precision=precision, dumps=True) for _, job in stream]
        results = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(stream) and st["failed"] == 0
    for (_, job), got, ref in zip(stream, results, refs):
        name = job["name"]
        # equal categories share one system per node: the library's slot n
        # is the oracle's slot n*K (category 0)
        K = len(ref["status"]) // len(got["status"])
        cap = ref["cap"]
        r_status = ref["status"][::K]
        r_count = ref["nb_count"][::K]
        r_index = ref["nb_index"].reshape(-1, cap)[::K]
        r_var = ref["variance"][::K]
        assert np.array_equal(got["status"], r_status), name
        kriged = r_status >= 0  # informed cells of OK/SK have no system (and no list)
        assert np.array_equal(got["nb_count"][kriged], r_count[kriged]), name
        valid = (np.arange(cap)[None, :] < np.maximum(r_count, 0)[:, None]) & kriged[:, None]
        gi = got["nb_index"].reshape(-1, got["cap"])[:, :cap]
        assert np.array_equal(gi[valid], r_index[valid]), name
        assert np.array_equal(got["out_mask"], ref["out_mask"]), name
        ok = r_status == 0
        sill = job["params"][0]["sill"]
        if job["kind"] == "ik":
            assert np.array_equal(got["out"], ref["out"]), name
        elif precision == "fp64":
            assert np.array_equal(got["out"].view(np.uint32), ref["out"].view(np.uint32)), name
        else:
            informed = job["mask"] > 0
            scale = float(np.max(np.abs(job["values"][informed])))
            assert rel_err(got["out"], ref["out"], 1e-6 * scale).max() <= 1e-6, name
        if precision == "fp64":
            assert np.array_equal(got["variance"][ok].view(np.uint64), r_var[ok].view(np.uint64)), name
        else:
            assert rel_err(got["variance"][ok], r_var[ok], 1e-6 * sill).max() <= 1e-6, name
