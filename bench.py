"""Benchmark of the kriging path on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): simple kriging of the 256x256x64 synthetic cube, 1 %
informed cells from an FFT Gaussian field, exponential variogram (40,20,8)
azimuth 30, sill 1, nugget 0.05, radii (80,40,16), 32 neighbours, SK mean 0
(hpgl_b200.workloads.sk_ok_256x256x64) — every uninformed node kriged once.
Metric: kriged nodes/s.

* ``value``: FP32 factorisation + FP64 refinement, device-resident (inputs
  in HBM before the timed region; each step re-runs search, covariance
  build, solve and estimate), CUDA events on the library's stream, 256 MiB
  written between steps to flush L2; whole job = all ranks' nodes / max rank
  time.  ``fp64`` holds the same for the bit-exact FP64 path and
  ``mixed_vs_fp64`` their ratio.
* ``e2e``: the same metric through the public C ABI (hpgl_b200_krige) from
  host buffers: planning, host->device copies, device work and device->host
  copies of the estimate and mask inside each timed call.
* ``cpu_baseline``: the reference's own simple kriging (compiled from its
  sources by oracle/build_ref.sh) through its stock entry point
  hpgl_simple_kriging on the whole job, all host threads (2 timed calls).
* ``--impl reference``: that reference CPU path as the timed arm, one whole
  job per step.

``--workload inc_io``: the INC property file reader and writer instead
(hpgl_b200/bench_io.py), with the reference's own reader and writer beside;
``--workload variogram``: experimental variograms (hpgl_b200/bench_variogram.py);
``--workload sgs``: sequential Gaussian and indicator simulation
(hpgl_b200/bench_sim.py); ``--workload cokriging``: colocated simple
cokriging, Markov models I and II (hpgl_b200/bench_cok.py); ``--workload
configs``: every kriging configuration, mixed and FP64 (hpgl_b200/bench_configs.py);
``--workload serve_jobs``: the serving stream's jobs each alone
(hpgl_b200/bench_serve_jobs.py; ``--job``, ``--crop`` for profiling).

Multi-GPU: the path has no exchange step; N ranks (torchrun, one per GPU)
each krige their own copy of the job ("replicas only", weak scaling).
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "kriged nodes/s"
WORKLOAD = "sk_256x256x64_exp(40,20,8)_az30_r(80,40,16)_n32_1pct"


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_flops(nb_counts, rhs):
    """Per-system work of the path: F(N) = 2/3 N^3 (Cholesky) + 2 R N^2
    (triangular solves) + 4N (combine, variance), plus 20 flop for each of the
    N(N+1)/2 + N covariance entries; summed over the kriged systems."""
    n = nb_counts.astype(np.float64)
    f = 2.0 / 3.0 * n ** 3 + 2.0 * rhs * n ** 2 + 4.0 * n + 20.0 * (n * (n + 1) / 2.0 + n)
    return float(f.sum())


def cpu_reference(job, steps, warmup, threads):
    """The reference's own simple kriging through its stock C entry point
    hpgl_simple_kriging (compiled from its sources into oracle/_ref; the
    per-node progress tick of cont_kriging.h:108-111 included) on the whole
    job, `threads` OpenMP threads.  Returns (nodes/s per timed call, kind,
    description, threads used).  Without the reference build, the oracle
    restatement runs the same job ("port")."""
    from oracle import oracle as O
    kriged = int((job["mask"] == 0).sum())
    if O.reference_available():
        r = O.RefSimpleKriging(job, threads)
        call, used, kind = r.call, r.threads, "reference"
    else:
        def call():
            O.run(job, dumps=False, threads=threads)
        used, kind = threads, "port"
    rates = []
    for it in range(warmup + steps):
        t = time.perf_counter()
        call()
        dt = time.perf_counter() - t
        if it >= warmup:
            rates.append(kriged / dt)
    desc = ("the whole job (%d kriged nodes) per call through hpgl_simple_kriging, %d OpenMP threads"
            % (kriged, used))
    return rates, kind, desc, used


def run_reference_arm(args):
    world, rank, _ = _dist()
    if rank != 0:
        return 0
    from hpgl_b200 import workloads as W
    job = W.sk_ok_256x256x64()
    kriged = int((job["mask"] == 0).sum())
    threads = os.cpu_count() or 1
    # one whole job per step takes seconds on the host cores: one untimed
    # call warms the library (page faults, thread pool) and keeps the run
    # within a few minutes
    warm = min(args.warmup, 1)
    rates, kind, desc, used = cpu_reference(job, args.steps, warm, threads)
    v = float(np.median(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "nodes/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": warm, "ms_per_step": 1000.0 * kriged / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": list(job["shape"]), "kriged_nodes_per_step": kriged,
                   "entry": "hpgl_simple_kriging", "sample": desc},
        "cpu_baseline": {"value": v, "unit": "nodes/s", "cores": used, "kind": kind, "sample": desc},
        "e2e": {"value": v, "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-jobs", type=int, default=40)
    ap.add_argument("--serve-rates", default="5,20,50,100,200", help="arrival rates (jobs/s) of the serving sweep")
    ap.add_argument("--grid", default=None, help="NXxNYxNZ: same workload on another grid (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch setting (profiling runs)")
    ap.add_argument("--job", default=None, help="serve_jobs: keep the stream's job of this name")
    ap.add_argument("--crop", default=None, help="serve_jobs: NXxNYxNZ, cut the job's cube (profiling runs)")
    ap.add_argument("--workload", default="krige",
                    choices=["krige", "inc_io", "variogram", "sgs", "cokriging", "configs", "serve_jobs"],
                    help="inc_io: INC property file read/write (hpgl_b200/bench_io.py); variogram: experimental "
                         "variograms (hpgl_b200/bench_variogram.py); sgs: sequential Gaussian and indicator "
                         "simulation (hpgl_b200/bench_sim.py); cokriging: colocated simple cokriging "
                         "(hpgl_b200/bench_cok.py); configs: every kriging configuration "
                         "(hpgl_b200/bench_configs.py); serve_jobs: the serving stream's jobs each alone "
                         "(hpgl_b200/bench_serve_jobs.py); one GPU")
    args = ap.parse_args()
    if args.workload == "inc_io":
        from hpgl_b200 import bench_io
        return bench_io.run(args, ROOT)
    if args.workload == "variogram":
        from hpgl_b200 import bench_variogram
        return bench_variogram.run(args, ROOT)
    if args.workload == "sgs":
        from hpgl_b200 import bench_sim
        return bench_sim.run(args, ROOT)
    if args.workload == "cokriging":
        from hpgl_b200 import bench_cok
        return bench_cok.run(args, ROOT)
    if args.workload == "configs":
        from hpgl_b200 import bench_configs
        return bench_configs.run(args, ROOT)
    if args.workload == "serve_jobs":
        from hpgl_b200 import bench_serve_jobs
        return bench_serve_jobs.run(args, ROOT)
    if args.impl == "reference":
        return run_reference_arm(args)
    args.warmup = max(args.warmup, 3)

    world, rank, local = _dist()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from hpgl_b200 import build
    from hpgl_b200 import native as N
    from hpgl_b200 import workloads as W
    if not os.path.exists(N.LIB_PATH):
        build.build()
    shape = tuple(int(v) for v in args.grid.split("x")) if args.grid else (256, 256, 64)
    job = W.sk_ok_256x256x64(shape=shape)
    size = int(np.prod(job["shape"]))
    kriged = int((job["mask"] == 0).sum())

    from replicas import barrier, max_over_ranks, whole_job_rate

    # Untimed run of each path first (library warm-up, neighbour counts).
    dump = N.krige(job, precision="fp64", dumps=True)
    nbc = dump["nb_count"][dump["status"] >= 0]
    flops = algorithmic_flops(nbc, rhs=1)
    del dump

    # Launch autotuning (our own tuner: fused vs separate search/solve and
    # persistent blocks per SM), untimed.
    tuning = {}
    for prec in ("mixed", "fp64"):
        if args.no_autotune:
            tuning[prec] = {"schedule": "split", "blocks_per_sm": 0, "candidates": 0}
            continue
        t = N.autotune(job, precision=prec)
        tuning[prec] = dict(t["chosen"], candidates=len(t["candidates"]))

    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    ms_mixed, info_m = N.bench(job, precision="mixed", iters=args.steps, warmup=args.warmup)
    clk = clocks.stop()
    barrier()
    ms_fp64, info_f = N.bench(job, precision="fp64", iters=args.steps, warmup=args.warmup)
    barrier()
    t_mixed = max_over_ranks(float(ms_mixed.sum()))
    t_fp64 = max_over_ranks(float(ms_fp64.sum()))
    value = whole_job_rate(world, kriged * args.steps, t_mixed)
    fp64_value = whole_job_rate(world, kriged * args.steps, t_fp64)

    # End to end through the public API from host buffers, both precisions;
    # the library reports each call's split (planning, copies, device).
    e2e = {}
    for prec in ("mixed", "fp64"):
        N.krige(job, precision=prec)
        barrier()
        parts = {k: [] for k in ("ms_total", "ms_plan", "ms_h2d", "ms_device", "ms_d2h")}
        for _ in range(args.steps):
            r = N.krige(job, precision=prec)
            for k in parts:
                parts[k].append(r[k])
        t_e2e = max_over_ranks(float(np.sum(parts["ms_total"])))
        e2e[prec] = dict(value=whole_job_rate(world, kriged * args.steps, t_e2e), ms_per_step=t_e2e / args.steps,
                         split_ms={k[3:]: float(np.mean(v)) for k, v in parts.items() if k != "ms_total"})
    h2d = size * 4 + size * 1
    d2h = size * 4 + size * 1

    # Per-result error of the mixed path against the FP64 path (bit-identical
    # to the reference's arithmetic): every kriged node's estimate and
    # kriging variance, untimed.
    ref64 = N.krige(job, precision="fp64", dumps="variance")
    mix = N.krige(job, precision="mixed", dumps="variance")
    okv = ref64["status"] == 0
    scale = float(np.max(np.abs(job["values"][job["mask"] > 0])))
    sill = job["params"][0]["sill"]
    err_est = np.abs(mix["out"].astype(np.float64) - ref64["out"]) / np.maximum(np.abs(ref64["out"]), 1e-6 * scale)
    err_var = np.abs(mix["variance"][okv] - ref64["variance"][okv]) / np.maximum(np.abs(ref64["variance"][okv]),
                                                                                  1e-6 * sill)
    mixed_error = {"max_rel_err_estimate": float(err_est.max()), "max_rel_err_variance": float(err_var.max()),
                   "tolerance": 1e-6, "floors": "1e-6 x max |informed value| (estimates), 1e-6 x sill (variances)",
                   "nodes": int(okv.sum()), "statuses_equal": bool(np.array_equal(ref64["status"], mix["status"])),
                   "masks_equal": bool(np.array_equal(ref64["out_mask"], mix["out_mask"]))}
    del ref64, mix

    # Roofline of the dominant kernel (the solve): algorithmic flops per
    # launch / CUDA-event duration, against the FP32 CUDA-core rate measured
    # here by an FMA-loop kernel timed alone (hpgl_b200_fma_peak; the
    # measured-peaks file holds HBM and bf16-tensor figures only).
    peak_fp32 = N.fma_peak("mixed")
    peak_fp64 = N.fma_peak("fp64")
    achieved = flops / (info_m["ms_top_kernel"] / 1000.0) / 1e12
    achieved64 = flops / (info_f["ms_top_kernel"] / 1000.0) / 1e12
    traffic = None
    try:
        tj = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))[info_m["top_kernel"]]
        # measured on the 128x128x32 cube; DRAM traffic scales with the systems
        traffic = tj["dram_bytes_per_launch_128x128x32"] * kriged / tj["systems_128x128x32"]
    except (OSError, KeyError, ValueError):
        pass
    roofline = {"kernel": info_m["top_kernel"], "bound": "fp32", "achieved": achieved, "peak": peak_fp32,
                "unit": "TFLOP/s", "frac": achieved / peak_fp32, "traffic": traffic, "traffic_unit": "bytes/launch",
                "peak_source": "measured FP32 CUDA-core rate, FMA-loop kernel timed alone (hpgl_b200_fma_peak)",
                "ms_per_launch": info_m["ms_top_kernel"], "flop_per_launch": flops,
                "fp64_solve": {"kernel": info_f["top_kernel"], "achieved": achieved64, "peak": peak_fp64,
                               "frac": achieved64 / peak_fp64, "ms_per_launch": info_f["ms_top_kernel"]}}

    # Serving: Poisson streams of mixed OK/SK/IK jobs (grids 32^3 ..
    # 256x256x64, ranges 5-60, 8-64 neighbours) replayed in real time
    # against the continuous-batching server at each arrival rate; p50/p99
    # submit-to-completion latency, systems/s and where a job's time went.
    # The same jobs run back to back through the synchronous call give the
    # batch rate the stream is compared with.
    serve = None
    if not args.no_serve:
        from hpgl_b200 import serve as SV
        rates = [float(r) for r in args.serve_rates.split(",")]
        serve = {"jobs_per_rate": args.serve_jobs, "hbm_budget_gb": 120, "max_inflight": 8, "rates": []}
        batch_stream = W.serve_stream(args.serve_jobs, 1.0, seed=5 + rank)
        for prec in ("mixed", "fp64"):
            t = time.perf_counter()
            systems = 0
            for _, sjob in batch_stream:
                systems += N.krige(sjob, precision=prec)["systems"]
            serve["batch_" + prec] = {"systems_per_s": systems / (time.perf_counter() - t),
                                      "note": "the same jobs back to back through hpgl_b200_krige (whole calls)"}
        for rate in rates:
            stream = W.serve_stream(args.serve_jobs, rate, seed=5 + rank)
            row = {"rate_jobs_per_s": rate}
            for prec in ("mixed", "fp64"):
                st, _ = SV.run_stream(stream, precision=prec, hbm_budget_bytes=120 << 30, max_inflight=8)
                row[prec] = {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "systems_per_s": st["systems_per_s"],
                             "completed": st["completed"], "failed": st["failed"],
                             "peak_inflight": st["peak_inflight"],
                             "mean_split_ms": {"plan": st["mean_plan_ms"], "admission_wait": st["mean_wait_ms"],
                                               "device_and_copies": st["mean_run_ms"]}}
            serve["rates"].append(row)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rates, kind, desc, used = cpu_reference(job, 2, 1, threads)
        cpu = {"value": float(np.median(rates)), "unit": "nodes/s", "cores": used, "kind": kind,
               "sample": desc}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "nodes/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_mixed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": list(job["shape"]), "kriged_nodes_per_step": kriged,
                       "precision": "fp32 factorisation + fp64 refinement, fp64 re-solve of routed systems",
                       "l2": "256 MiB written between steps", "parallelism": "replicas%d" % world,
                       "launch": tuning, "pass": "one CUDA graph per step"},
            "fp64": {"value": fp64_value, "ms_per_step": t_fp64 / args.steps,
                     "top_kernel_ms": info_f["ms_top_kernel"]},
            "mixed_vs_fp64": value / fp64_value,
            "routed_to_fp64": info_m["systems_fp64"] / max(1, info_m["systems"]),
            "e2e": {"value": e2e["mixed"]["value"], "unit": "nodes/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e["mixed"]["ms_per_step"],
                    "split_ms": e2e["mixed"]["split_ms"],
                    "fp64": e2e["fp64"]},
            "mixed_error": mixed_error,
            "roofline": roofline,
            "clocks": clk,
            "gpu_launches": info_m["launches"] * args.steps,
            "cpu_baseline": cpu,
            "serve": serve,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
