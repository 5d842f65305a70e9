"""Benchmark of the experimental variograms (``python bench.py --workload variogram``).

Grid workload: the 166 x 141 x 225 cube (5,266,350 cells, the cube of the
reference's published kriging timings) with 10 % informed cells, values
N(0,1) plus a trend; a horizontal tunnel along azimuth 30 (R2 = 4, R3 = 2,
tolerance 0.8), 20 lags of width and separation 2.  Unit: candidate pairs
(tunnel offsets x informed cells) per second, the work the reference's loop
does per informed cell.

Point-set workload: 20 000 points in a 1000 x 1000 x 50 box (well-like
scatter), a horizontal tunnel along azimuth 320 (R2 = 500, R3 = 5, opening
0.8), 12 lags of 55 (the reference's lesson 5.2 template scaled to the box).
Unit: ordered point pairs per second.

* ``value``: the grid variogram's kernels (CUDA events around them inside
  the call, data and cell list already in HBM); ``e2e``: the whole C-ABI call
  from host arrays (copies, cell compaction, offsets, kernels, result).
* ``cpu_baseline``: the reference's own calc_variograms /
  calc_variograms_from_point_set (``oracle/_ref``, one thread, as it runs) on
  a smaller sample of the same workloads (a 166 x 141 x 20 slab; 4 000
  points), in the same unit.
"""

import json
import os
import time

import numpy as np

GRID = (166, 141, 225)
GRID_TEMPLATE = (2.0, 2.0, 0.8, 20, 0.0, (40.0, 4.0, 2.0), (30.0, 0.0, 0.0))
POINT_TEMPLATE = (55.0, 55.0, 0.8, 12, 0.0, (1.0, 500.0, 5.0), (320.0, 0.0, 0.0))


def grid_data(shape, seed=0):
    rng = np.random.default_rng(seed)
    x = np.arange(shape[0], dtype=np.float32)[:, None, None]
    v = np.asfortranarray((rng.normal(size=shape) + 0.02 * x).astype(np.float32))
    m = np.asfortranarray((rng.random(shape) < 0.10).astype(np.uint8))
    return v, m


def point_data(n, seed=1):
    rng = np.random.default_rng(seed)
    xs = (rng.random(n) * 1000).astype(np.float32)
    ys = (rng.random(n) * 1000).astype(np.float32)
    zs = (rng.random(n) * 50).astype(np.float32)
    vals = (rng.normal(size=n) + 0.001 * xs).astype(np.float32)
    return {"X": xs, "Y": ys, "Z": zs, "Property": vals}


def _template(CV, spec):
    ell = CV.Ellipsoid(spec[5][0], spec[5][1], spec[5][2], spec[6][0], spec[6][1], spec[6][2])
    return CV.VariogramSearchTemplate(spec[0], spec[1], spec[2], spec[3], spec[4], ell)


def _timed(f, steps, warmup):
    for _ in range(warmup):
        f()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        f()
        ts.append((time.perf_counter() - t0) * 1e3)
    return float(np.median(ts))


def run(args, root):
    from hpgl_b200 import cvariogram as CV
    from hpgl_b200.geo_bsd import geo
    from oracle import oracle as O
    v, m = grid_data(GRID)
    t = _template(CV, GRID_TEMPLATE)
    ninf = int(m.sum())

    dev = []

    def grid_call():
        CV.CalcVariograms(t, (v, m))
        dev.append(geo.io_last_timing()["ms_device"])

    ms_grid = _timed(grid_call, args.steps, max(args.warmup, 1))
    ms_grid_dev = float(np.median(dev[-args.steps:]))
    grid_pairs = int(geo.io_last_timing()["tokens"])  # tunnel offsets with a lag x informed cells
    noff = grid_pairs // ninf
    pts = point_data(20000)
    tp = _template(CV, POINT_TEMPLATE)
    n = pts["X"].size

    pdev = []

    def point_call():
        CV.CalcVariogramsFromPointSet(tp, pts)
        pdev.append(geo.io_last_timing()["ms_device"])

    ms_points = _timed(point_call, args.steps, max(args.warmup, 1))
    ms_points_dev = float(np.median(pdev[-args.steps:]))

    cpu = None
    if not args.no_cpu_baseline and O.reference_cv_available():
        slab = (GRID[0], GRID[1], 20)
        sv, sm = grid_data(slab, seed=2)
        ot = O.cv_template(*GRID_TEMPLATE)
        t0 = time.perf_counter()
        O.ref_variograms(ot, sv, sm)
        ref_grid_s = time.perf_counter() - t0
        ref_grid_rate = noff * int(sm.sum()) / ref_grid_s
        sp = point_data(4000, seed=3)
        op = O.cv_template(*POINT_TEMPLATE)
        t0 = time.perf_counter()
        O.ref_variograms_points(op, sp["X"], sp["Y"], sp["Z"], sp["Property"])
        ref_pt_s = time.perf_counter() - t0
        ref_pt_rate = 4000.0 * 4000.0 / ref_pt_s
        cpu = {"kind": "reference", "cores": 1,
               "sample": "166x141x20 slab of the grid workload; 4000 points of the point-set workload",
               "value": ref_grid_rate, "unit": "pairs/s", "grid_pairs_per_s": ref_grid_rate,
               "points_pairs_per_s": ref_pt_rate, "grid_s": ref_grid_s, "points_s": ref_pt_s}
    line = {
        "metric": "variogram pairs/s", "value": grid_pairs / (ms_grid_dev / 1e3), "unit": "pairs/s", "n_gpus": 1,
        "ms_device": ms_grid_dev,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32 values, f64 sums",
        "data": "synthetic",
        "config": {"workload": "variogram_grid_166x141x225_10pct_20lags+points_20000_12lags",
                   "tunnel_offsets": noff, "informed_cells": ninf, "grid_pairs": grid_pairs,
                   "point_pairs": n * n},
        "e2e": {"value": grid_pairs / (ms_grid / 1e3), "unit": "pairs/s", "ms": ms_grid,
                "h2d_bytes_per_step": int(v.nbytes + m.nbytes), "d2h_bytes_per_step": 4 * GRID_TEMPLATE[3]},
        "points": {"value": n * n / (ms_points_dev / 1e3), "unit": "pairs/s", "ms_device": ms_points_dev,
                   "e2e": n * n / (ms_points / 1e3), "ms": ms_points},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    return 0
