"""Benchmark of the INC property files (``python bench.py --workload inc_io``).

Workload: a 166 x 141 x 225 continuous property (5,266,350 cells, the cube
the reference's SK / OK / IK timings are quoted on), lognormal values of
both signs with 20 % of the cells undefined (-99), written as an INC file
(one "%E" line per cell, 70 MB) and read back.  Metric: values/s.

* ``read`` / ``write``: through the C ABI (hpgl_read_inc_file_float,
  hpgl_write_inc_file_float) from and to host buffers and the page cache:
  file read or write, copies and kernels inside each timed call (e2e).
* ``device``: the kernels alone (CUDA events around the device passes of
  the same calls); the roofline uses their algorithmic bytes — text read
  once plus 5 B per value written for the reader, cells read (5 B) plus
  text written for the writer — over the measured HBM copy bandwidth.
* ``reference``: the reference's own reader and writer (oracle/_ref, one
  thread, as the reference runs them) on the same files.
"""

import ctypes as C
import json
import os
import tempfile
import time

import numpy as np

SHAPE = (166, 141, 225)
UNDEF = -99.0


def property_cells(seed=0):
    n = int(np.prod(SHAPE))
    rng = np.random.default_rng(seed)
    v = (rng.lognormal(-1.5, 0.8, n) * np.where(rng.random(n) < 0.5, 1, -1)).astype(np.float32)
    v[rng.random(n) < 0.2] = UNDEF
    m = (v != UNDEF).astype(np.uint8)
    return v, m


def _hbm_peak(root):
    try:
        j = json.load(open(os.path.join(root, "MEASURED_PEAKS.json")))
        for k in ("hbm_gbs", "hbm_GBs", "hbm_copy_gbs"):
            if k in j:
                return float(j[k]), "measured"
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback"


def run(args, root):
    from hpgl_b200.geo_bsd import geo
    from hpgl_b200.geo_bsd import hpgl_wrap as W
    so = W._hpgl_so
    v, m = property_cells()
    n = v.size
    d = tempfile.mkdtemp(prefix="inc_io_", dir=os.environ.get("TMPDIR", "/tmp"))
    path = os.path.join(d, "poro.inc")
    sh = W._HPGL_SHAPE()
    sh.data[:] = (n, 1, 1)
    arr = W._HPGL_CONT_MASKED_ARRAY(data=v.ctypes.data_as(C.POINTER(C.c_float)),
                                    mask=m.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh)
    out_v = np.zeros(n, np.float32)
    out_m = np.zeros(n, np.uint8)

    def write_once():
        so.hpgl_write_inc_file_float(os.fsencode(path), C.byref(arr), UNDEF, b"PORO")
        W.check_last_error()
        return geo.io_last_timing()

    def read_once():
        so.hpgl_read_inc_file_float(os.fsencode(path), UNDEF, n, out_v, out_m)
        W.check_last_error()
        return geo.io_last_timing()

    for _ in range(args.warmup):
        write_once()
        read_once()
    wt, rt = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        tw = write_once()
        tw["wall_ms"] = (time.perf_counter() - t0) * 1e3
        wt.append(tw)
        t0 = time.perf_counter()
        tr = read_once()
        tr["wall_ms"] = (time.perf_counter() - t0) * 1e3
        rt.append(tr)
    text_bytes = os.path.getsize(path)
    # "%E" keeps 7 significant digits: the values come back within half a unit of the 7th
    assert np.array_equal(out_m, m) and np.allclose(out_v[m > 0], v[m > 0], rtol=6e-7, atol=0)

    def med(ts, k):
        return float(np.median([t[k] for t in ts]))

    peak, src = _hbm_peak(root)
    read_dev_ms, write_dev_ms = med(rt, "ms_device"), med(wt, "ms_device")
    read_bytes = text_bytes + 5 * n
    write_bytes = 5 * n + text_bytes
    roof_read = read_bytes / (read_dev_ms / 1e3) / 1e9
    roof_write = write_bytes / (write_dev_ms / 1e3) / 1e9

    ref = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.reference_available():
            rv = np.zeros(n, np.float32)
            rm = np.zeros(n, np.uint8)
            rpath = os.path.join(d, "ref.inc")
            t0 = time.perf_counter()
            O.ref_write_prop(rpath, "PORO", v, m, UNDEF)
            ref_write_ms = (time.perf_counter() - t0) * 1e3
            t0 = time.perf_counter()
            rv, rm = O.ref_read_inc(path, n, UNDEF)
            ref_read_ms = (time.perf_counter() - t0) * 1e3
            same_file = open(rpath, "rb").read() == open(path, "rb").read()
            ref = {"kind": "reference", "cores": 1, "sample": "the whole file, one call each",
                   "read_values_per_s": n / (ref_read_ms / 1e3), "write_values_per_s": n / (ref_write_ms / 1e3),
                   "read_ms": ref_read_ms, "write_ms": ref_write_ms, "same_file": same_file,
                   "same_values": bool(np.array_equal(rv.view(np.uint8), out_v.view(np.uint8)))}
    os.remove(path)
    try:
        os.remove(os.path.join(d, "ref.inc"))
    except OSError:
        pass
    os.rmdir(d)
    line = {
        "metric": "INC values read/s", "value": n / (read_dev_ms / 1e3), "unit": "values/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "u8 text -> f32",
        "data": "synthetic", "config": {"workload": "inc_read_write_166x141x225_E_format", "cells": n,
                                        "text_bytes": text_bytes, "undefined_fraction": 0.2},
        "e2e": {"value": n / (med(rt, "ms_total") / 1e3), "unit": "values/s", "ms": med(rt, "ms_total"),
                "h2d_bytes_per_step": text_bytes, "d2h_bytes_per_step": 5 * n},
        "read": {k: med(rt, k) for k in ("ms_file", "ms_h2d", "ms_device", "ms_d2h", "ms_total", "wall_ms")},
        "write": {k: med(wt, k) for k in ("ms_file", "ms_h2d", "ms_device", "ms_d2h", "ms_total", "wall_ms")},
        "write_values_per_s_e2e": n / (med(wt, "ms_total") / 1e3),
        "write_values_per_s_device": n / (write_dev_ms / 1e3),
        "roofline": {"bound": "hbm", "unit": "GB/s", "peak": peak, "peak_source": src,
                     "read": {"achieved": roof_read, "frac": roof_read / peak, "bytes": read_bytes},
                     "write": {"achieved": roof_write, "frac": roof_write / peak, "bytes": write_bytes}},
        "cpu_baseline": ref,
    }
    print(json.dumps(line))
    return 0
