"""Benchmark of every kriging configuration (``python bench.py --workload configs``).

The four kriging cases of hpgl_b200.workloads.CONFIGS on their full grids:
ordinary kriging 50x50x20 (12 neighbours), simple and ordinary kriging
256x256x64 (32 neighbours), 4-category indicator kriging 200x200x100 (24
neighbours, one shared system per node: the four variograms are equal),
LVM kriging 512x512x32 (64 neighbours).  Per case: the device pass (CUDA
events, inputs in HBM, 256 MiB written between passes, one CUDA-graph
replay per pass) for the FP32-refined path and for plain FP64, the share
of systems the mixed path re-solved in FP64, and whole hpgl_b200_krige calls
from host buffers (median of three after one warm-up call).  Unit: kriged systems per second (IK counts a
system per category, as the reference solves one per category).
"""

import json
import time

import numpy as np


def _case(name, job, kind, N, steps, warmup):
    out = {"kind": kind}
    for precision in ("mixed", "fp64"):
        ms, info = N.bench(job, precision=precision, iters=steps, warmup=warmup, kind=kind)
        systems = info["systems"]
        out[precision] = {"ms": float(np.median(ms)), "systems_per_s": systems / (float(np.median(ms)) / 1e3),
                          "top_kernel": info["top_kernel"], "ms_top_kernel": info["ms_top_kernel"]}
        if precision == "mixed":
            out["systems"] = int(systems)
            out["rerouted_to_fp64"] = (info["systems_fp64"] / systems) if systems else 0.0
    # whole calls from host buffers: one warm-up (first-use costs: pinned
    # staging, arena growth, module loading), then the median of three
    N.krige(job, precision="mixed", kind=kind)
    calls = []
    for _ in range(3):
        t0 = time.perf_counter()
        N.krige(job, precision="mixed", kind=kind)
        calls.append((time.perf_counter() - t0) * 1e3)
    out["e2e_ms"] = float(np.median(calls))
    out["e2e_systems_per_s"] = out["systems"] / (out["e2e_ms"] / 1e3)
    out["mixed_vs_fp64"] = out["fp64"]["ms"] / out["mixed"]["ms"]
    return out


def run(args, root):
    from hpgl_b200 import native as N
    from hpgl_b200 import workloads as W
    steps, warmup = max(args.steps, 1), max(args.warmup, 3)
    cases = {}
    for name, kind in (("ok_50x50x20", "ok"), ("sk_ok_256x256x64", "sk"), ("sk_ok_256x256x64", "ok"),
                       ("ik_200x200x100", "ik"), ("lvm_512x512x32", "lvm")):
        job = W.CONFIGS[name]()
        cases["%s:%s" % (name, kind)] = _case(name, job, kind, N, steps, warmup)
    first = cases["ik_200x200x100:ik"]
    line = {
        "metric": "kriged systems/s", "value": first["mixed"]["systems_per_s"], "unit": "systems/s", "n_gpus": 1,
        "steps": steps, "warmup": warmup, "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": "ik_200x200x100 (value) and every configuration (cases)",
                   "l2": "256 MiB written between passes"},
        "cases": cases,
    }
    print(json.dumps(line))
    return 0
