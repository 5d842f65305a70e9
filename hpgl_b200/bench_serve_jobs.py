"""Per-job timing of the serving stream (``python bench.py --workload serve_jobs``).

The jobs of hpgl_b200.workloads.serve_stream (40 jobs, seed 5: grids
log-uniform between 32^3 and 256x256x64, 0.5-3 % informed, spherical /
exponential / Gaussian variograms with ranges 5-60, 8-64 neighbours, OK / SK
/ 4-category IK), each run alone: the device pass (CUDA events, inputs in
HBM, one CUDA-graph replay per pass) in the FP32-refined and plain FP64
precisions, with its search and top-kernel times, the systems solved and the
share re-solved in FP64.  Shows which jobs the stream's device time goes to.

``--job NAME`` keeps one job (e.g. serve_31); ``--crop NXxNYxNZ`` cuts its
cube to the first NX x NY x NZ cells with the same variogram and search
(small cases of the same kernels for profiling captures).
"""

import json

import numpy as np


def _crop(job, dims):
    nx, ny, nz = job["shape"]
    sx, sy, sz = (min(a, b) for a, b in zip(dims, (nx, ny, nz)))

    def cut(a):
        return np.ascontiguousarray(a.reshape((nx, ny, nz), order="F")[:sx, :sy, :sz]).reshape(-1, order="F")

    out = dict(job, shape=(sx, sy, sz), name="%s_%dx%dx%d" % (job["name"], sx, sy, sz))
    for k in ("mask", "values", "codes"):
        if k in job:
            out[k] = cut(job[k])
    return out


def run(args, root):
    from hpgl_b200 import native as N
    from hpgl_b200 import workloads as W
    stream = W.serve_stream(args.serve_jobs, 1.0, seed=5)
    jobs = [j for _, j in stream if args.job is None or j["name"] == args.job]
    if not jobs:
        raise SystemExit("no job named %r in the stream" % args.job)
    steps, warmup = max(1, args.steps), max(0, args.warmup)
    rows = []
    for job in jobs:
        if args.crop:
            job = _crop(job, tuple(int(v) for v in args.crop.lower().split("x")))
        p = job["params"][0]
        row = {"job": job["name"], "kind": job["kind"], "grid": list(job["shape"]), "cov_type": p["cov_type"],
               "radii": list(p["radii"]), "max_neighbours": p["max_neighbours"]}
        for precision in ("mixed", "fp64"):
            ms, info = N.bench(job, precision=precision, iters=steps, warmup=warmup, flush_bytes=0)
            row[precision] = {"ms": float(np.median(ms)), "ms_search": info["ms_search"],
                              "top_kernel": info["top_kernel"], "ms_top_kernel": info["ms_top_kernel"],
                              "ms_resolve": info["ms_resolve"], "systems": int(info["systems"]),
                              "share_fp64": (info["systems_fp64"] / info["systems"]) if info["systems"] else 0.0}
        rows.append(row)
        print(json.dumps(row), flush=True)
    total = {prec: sum(r[prec]["ms"] for r in rows) for prec in ("mixed", "fp64")}
    systems = sum(r["mixed"]["systems"] for r in rows)
    print(json.dumps({"metric": "kriged systems/s", "value": systems / (total["mixed"] / 1e3), "unit": "systems/s",
                      "n_gpus": 1, "steps": steps, "warmup": warmup, "higher_is_better": True, "dtype": "f32+f64",
                      "data": "synthetic",
                      "config": {"workload": "serving stream jobs, each alone (%d jobs%s%s)" % (
                          len(rows), ", job " + args.job if args.job else "", ", crop " + args.crop if args.crop else "")},
                      "device_ms_total": total, "systems": systems}))
    return 0
