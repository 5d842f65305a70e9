"""Benchmark of colocated simple cokriging (``python bench.py --workload cokriging``).

Workload: the 256 x 256 x 64 cube (4,194,304 cells) of the kriging benchmark,
a sparse primary property (2 % informed, a spherical Gaussian field) and a
dense correlated secondary one (90 % informed), spherical variogram of
ranges (14, 14, 5), radii (14, 14, 5), 32 neighbours, correlation 0.7
(hpgl_b200.workloads.cokriging_job): Markov model I, and Markov model II with
an exponential secondary model.  Unit: kriged nodes per second.

* ``value``: the device pass of Markov model I (template search and the
  cokriging systems in the reference's Gauss elimination order, FP64;
  inputs in HBM, CUDA events on the library's stream, 256 MiB written
  between passes); ``mm2`` the same for Markov model II.
* ``e2e``: the whole hpgl_b200_krige call from host buffers (planning,
  copies in, device work, copies out).
* ``cpu_baseline``: the reference's own hpgl_simple_cokriging_mark1 / _mark2
  (``oracle/_ref``, compiled from its sources; single-threaded, as its
  cokriging is) on the 64 x 64 x 32 cube of the same workload.
``--grid NXxNYxNZ`` runs the same workload on another grid (profiling runs).
"""

import json
import time

import numpy as np

GRID = (256, 256, 64)
REF_GRID = (64, 64, 32)


def _kriged(job):
    return int((np.asarray(job["mask"]) == 0).sum())


def run(args, root):
    from hpgl_b200 import native as N
    from hpgl_b200 import workloads as W
    from oracle import oracle as O
    grid = tuple(int(v) for v in args.grid.split("x")) if args.grid else GRID
    steps, warmup = max(args.steps, 1), max(args.warmup, 3)
    out = {}
    for mark in (1, 2):
        job = W.cokriging_job(shape=grid, mark=mark, max_neighbours=32)
        n = _kriged(job)
        ms, info = N.bench(job, precision="fp64", iters=steps, warmup=warmup)
        walls = []
        for _ in range(warmup):
            N.krige(job, precision="fp64")
        for _ in range(steps):
            t0 = time.perf_counter()
            N.krige(job, precision="fp64")
            walls.append((time.perf_counter() - t0) * 1e3)
        out[mark] = dict(nodes=n, ms=float(np.median(ms)), top_kernel=info["top_kernel"],
                         ms_top_kernel=info["ms_top_kernel"], e2e_ms=float(np.median(walls)),
                         h2d=int(job["values"].nbytes * 2 + job["mask"].nbytes * 2),
                         d2h=int(job["values"].nbytes + job["mask"].nbytes))
    cpu = None
    if not args.no_cpu_baseline and O.reference_available():
        rates = {}
        for mark in (1, 2):
            rj = W.cokriging_job(shape=REF_GRID, mark=mark, max_neighbours=32)
            t0 = time.perf_counter()
            O.ref_cokriging(rj)
            rates[mark] = _kriged(rj) / (time.perf_counter() - t0)
        cpu = {"kind": "reference", "cores": 1, "sample": "the same workload on the %dx%dx%d cube" % REF_GRID,
               "value": rates[1], "unit": "nodes/s", "mm2_nodes_per_s": rates[2]}
    m1, m2 = out[1], out[2]
    line = {
        "metric": "kriged nodes/s", "value": m1["nodes"] / (m1["ms"] / 1e3), "unit": "nodes/s", "n_gpus": 1,
        "steps": steps, "warmup": warmup, "ms_per_step": m1["ms"], "higher_is_better": True, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "cok1_%dx%dx%d_n32" % grid, "kriged_nodes_per_step": m1["nodes"],
                   "top_kernel": m1["top_kernel"], "ms_top_kernel": m1["ms_top_kernel"],
                   "l2": "256 MiB written between passes"},
        "e2e": {"value": m1["nodes"] / (m1["e2e_ms"] / 1e3), "unit": "nodes/s", "ms": m1["e2e_ms"],
                "h2d_bytes_per_step": m1["h2d"], "d2h_bytes_per_step": m1["d2h"]},
        "mm2": {"value": m2["nodes"] / (m2["ms"] / 1e3), "ms_per_step": m2["ms"], "ms_top_kernel": m2["ms_top_kernel"],
                "e2e": m2["nodes"] / (m2["e2e_ms"] / 1e3), "e2e_ms": m2["e2e_ms"]},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    return 0
