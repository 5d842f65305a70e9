"""Benchmark of sequential simulation (``python bench.py --workload sgs``).

Workload: the reference's own large simulation test (its geo_testing
test_big_hard script): the 166 x 141 x 225 cube (5,266,350 cells) with 1 %
informed cells (seeded synthetic data in place of its BIG_HARD_DATA.INC,
which the reference does not ship), search radii (20, 20, 20), 12
neighbours, exponential variogram of ranges (10, 10, 10).

* SGS: values N(0, 1), sill 0.4 (the wrapper normalises it to 1), simple
  kriging, seed 3439275, the normal-score transform through the data's CDF
  (what the reference's sgs_simulation passes).
* SIS: two categories with marginal probabilities 0.8 / 0.2 (20 % of the
  informed codes are 1), the same variogram for both (median SIS), seed
  3241347; and (``sis4``, device time) the test's four categories: spherical
  ranges 4, 6, 2 and 10, sill 0.25, marginal probabilities 0.24, 0.235, 0.34
  and 0.18.

Unit: simulated nodes per second.  ``--grid NXxNYxNZ`` runs the same
workload on another grid (profiling runs).  ``value``: the simulation's device time
(CUDA events around the rounds; inputs in HBM); ``e2e``: the whole
geo_bsd.sgs_simulation call from host arrays (CDF transforms, path and
draws, copies, rounds, result).  ``cpu_baseline``: the reference's own
hpgl_sgs_simulation / hpgl_sis_simulation (``oracle/_ref``, compiled from
its sources; single-threaded, as its simulation is) on the same full
workload.
"""

import json
import time

import numpy as np

GRID = (166, 141, 225)
SGS_SEED = 3439275
SIS_SEED = 3241347


def _data(grid, seed=0):
    rng = np.random.default_rng(seed)
    n = int(np.prod(grid))
    values = rng.normal(size=n).astype(np.float32)
    mask = (rng.random(n) < 0.01).astype(np.uint8)
    codes = (rng.random(n) < 0.2).astype(np.uint8)
    return values, mask, codes


def _params(sill):
    return dict(cov_type=1, ranges=(10.0, 10.0, 10.0), angles=(0.0, 0.0, 0.0), sill=sill, nugget=0.0,
                radii=(20, 20, 20), max_neighbours=12)


def _timed(f, steps, warmup):
    out = None
    for _ in range(warmup):
        out = f()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        out = f()
        ts.append((time.perf_counter() - t0) * 1e3)
    return float(np.median(ts)), out


def run(args, root):
    from hpgl_b200 import native as N
    from hpgl_b200.geo_bsd import geo, sgs, sis
    from hpgl_b200.geo_bsd.cdf import calc_cdf
    from oracle import oracle as O
    GRID = tuple(int(v) for v in args.grid.split("x")) if args.grid else globals()["GRID"]
    values, mask, codes = _data(GRID)
    n = values.size
    nsim = int((mask == 0).sum())
    f = lambda a: np.asfortranarray(np.reshape(a, GRID, order="F"))
    grid = geo.SugarboxGrid(*GRID)
    prop = geo.ContProperty(f(values), f(mask))
    cdf = calc_cdf(prop)
    cov = geo.CovarianceModel(type=1, ranges=(10, 10, 10), sill=0.4)
    steps, warmup = max(args.steps, 1), max(args.warmup, 1)

    # SGS end to end through the Python entry point
    ms_sgs_e2e, out = _timed(lambda: sgs.sgs_simulation(prop, grid, cdf, (20, 20, 20), 12, cov, SGS_SEED), steps,
                             warmup)
    # device time of the same simulation (the normal-score values as input)
    gauss = O.cdf_transform(values, (cdf.values, cdf.probs), 0, mask)
    job = dict(shape=GRID, values=gauss, mask=mask, params=[_params(1.0)])
    dev = []
    rounds = tries = 0

    def sgs_dev():
        r = N.simulate(job, SGS_SEED, kind="sk")
        dev.append(r["ms_device"])
        return r

    _, r = _timed(sgs_dev, steps, warmup)
    ms_sgs_dev = float(np.median(dev[-steps:]))
    rounds, tries = r["rounds"], r["systems"]
    # where the time of one hpgl_b200_krige call goes (no CDF transforms)
    split = {k: round(float(r[k]), 2) for k in ("ms_plan", "ms_h2d", "ms_device", "ms_d2h", "ms_total")}

    # SIS
    ind = geo.IndProperty(f(codes), f(mask), 2)
    data = [{"cov_model": geo.CovarianceModel(type=1, ranges=(10, 10, 10), sill=1.0), "radiuses": (20, 20, 20),
             "max_neighbours": 12}] * 2
    ms_sis_e2e, _ = _timed(lambda: sis.sis_simulation(ind, grid, data, SIS_SEED, [0.8, 0.2]), steps, warmup)
    sis_params = [dict(_params(1.0), marginal_prob=0.8), dict(_params(1.0), marginal_prob=0.2)]
    sjob = dict(shape=GRID, codes=codes, mask=mask, values=None, kind="ik", params=sis_params)
    sdev = []

    def sis_dev():
        rr = N.simulate_indicator(sjob, SIS_SEED)
        sdev.append(rr["ms_device"])
        return rr

    _, rs = _timed(sis_dev, steps, warmup)
    ms_sis_dev = float(np.median(sdev[-steps:]))

    # four categories (the reference's multi-indicator case of the same test)
    rng4 = np.random.default_rng(4)
    probs4 = (0.24, 0.235, 0.34, 0.18)
    codes4 = rng4.choice(4, size=codes.size, p=np.array(probs4) / sum(probs4)).astype(np.uint8)
    sis4_params = [dict(_params(0.25), cov_type=0, ranges=(r, r, r), marginal_prob=q)
                   for r, q in zip((4.0, 6.0, 2.0, 10.0), probs4)]
    s4job = dict(shape=GRID, codes=codes4, mask=mask, values=None, kind="ik", params=sis4_params)
    s4dev = []

    def sis4_dev():
        rr = N.simulate_indicator(s4job, SIS_SEED)
        s4dev.append(rr["ms_device"])
        return rr

    _, rs4 = _timed(sis4_dev, steps, warmup)
    ms_sis4_dev = float(np.median(s4dev[-steps:]))

    cpu = None
    if not args.no_cpu_baseline and O.reference_available():
        t0 = time.perf_counter()
        O.ref_sgs(dict(shape=GRID, values=values, mask=mask, params=[_params(1.0)]), seed=SGS_SEED,
                  cdf=(cdf.values, cdf.probs))
        t_sgs = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.ref_sis(GRID, codes, mask, sis_params, seed=SIS_SEED)
        t_sis = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.ref_sis(GRID, codes4, mask, sis4_params, seed=SIS_SEED)
        t_sis4 = time.perf_counter() - t0
        cpu = {"kind": "reference", "cores": 1, "sample": "the full workload (SGS with the CDF transform; SIS)",
               "value": nsim / t_sgs, "unit": "nodes/s", "sgs_s": t_sgs, "sis_s": t_sis,
               "sis_nodes_per_s": nsim / t_sis, "sis4_s": t_sis4, "sis4_nodes_per_s": nsim / t_sis4}
    line = {
        "metric": "simulated nodes/s", "value": nsim / (ms_sgs_dev / 1e3), "unit": "nodes/s", "n_gpus": 1,
        "steps": steps, "warmup": warmup, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "ms_device": ms_sgs_dev,
        "config": {"workload": "sgs_%dx%dx%d_1pct_r20_n12_exp10+sis_2cat" % GRID, "simulated_nodes": nsim,
                   "rounds": rounds, "tries": tries, "ms_per_round": ms_sgs_dev / max(rounds, 1),
                   "call_split": split},
        "e2e": {"value": nsim / (ms_sgs_e2e / 1e3), "unit": "nodes/s", "ms": ms_sgs_e2e,
                "h2d_bytes_per_step": int(values.nbytes + mask.nbytes + cdf.values.nbytes + cdf.probs.nbytes),
                "d2h_bytes_per_step": int(values.nbytes + mask.nbytes)},
        "sis": {"value": nsim / (ms_sis_dev / 1e3), "ms_device": ms_sis_dev, "e2e": nsim / (ms_sis_e2e / 1e3),
                "ms": ms_sis_e2e, "rounds": rs["rounds"], "tries": rs["systems"]},
        "sis4": {"value": nsim / (ms_sis4_dev / 1e3), "ms_device": ms_sis4_dev, "rounds": rs4["rounds"],
                 "tries": rs4["systems"]},
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    return 0
