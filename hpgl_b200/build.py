"""Builds hpgl_b200/hpgl.so (the C-ABI library) for sm_100a.

    python -m hpgl_b200.build            # or hpgl_b200.build.build()

Device code: nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo.
Host planning code (plan.cpp) is built with -O2 -ffp-contract=off so its
covariance tables round exactly like the reference's arithmetic.  Objects go
to hpgl_b200/_build/, the library next to this file.  ptxas resource usage of
every kernel is written to hpgl_b200/_build/ptxas.log.
"""

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "hpgl.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
                   "-Xptxas", "-v", "-I", os.path.join(ROOT, "include")]
CXX_FLAGS = ["-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-Wall", "-Wno-unused-function",
             "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include"]

SOURCES_CU = ["kernels.cu", "solve32.cu", "solve64.cu", "cokriging.cu", "engine.cu", "sk_weights.cu", "textio.cu", "variogram.cu", "peak.cu"]
SOURCES_CXX = ["plan.cpp", "api.cpp", "sgs_host.cpp", "task_pool.cpp"]


def _run(cmd, log=None):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.append(r.stderr)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def _stale(obj, srcs):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "hpgl.h"))
    headers.append(os.path.join(ROOT, "include", "cvariogram.h"))
    jobs = []
    objs = []
    for f in SOURCES_CU:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([NVCC] + CU_FLAGS + ["-c", src, "-o", obj])
    for f in SOURCES_CXX:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
    logs = []
    with ThreadPoolExecutor(max_workers=4) as ex:
        for r in ex.map(lambda c: _run(c, logs), jobs):
            pass
    if jobs:
        with open(os.path.join(BUILD, "ptxas.log"), "w") as fh:
            fh.write("\n".join(logs))
    if force or jobs or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lpthread"])
        os.replace(tmp, LIB)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
