"""Continuous-batching kriging server (C ABI hpgl_b200_server_*) from Python.

    srv = Server(hbm_budget_bytes=120 << 30, max_inflight=8)
    t = srv.submit(job, precision="mixed")      # returns immediately
    out = srv.result(t)                          # waits; dict like native.krige
    srv.stats()                                  # p50/p99 ms, systems/s, ...

``run_stream(stream, ...)`` replays a list of (arrival_s, job) — e.g.
``workloads.serve_stream`` — submitting each job at its arrival time.
"""

import ctypes as C
import time

from . import native as N


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_longlong), ("max_inflight", C.c_int), ("worker_threads", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
                ("systems", C.c_longlong), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("wall_s", C.c_double), ("systems_per_s", C.c_double), ("peak_inflight", C.c_int),
                ("peak_bytes", C.c_longlong), ("mean_plan_ms", C.c_double), ("mean_wait_ms", C.c_double),
                ("mean_run_ms", C.c_double)]


def _bind():
    L = N.lib()
    if not getattr(L, "_server_bound", False):
        L.hpgl_b200_server_create.restype = C.c_void_p
        L.hpgl_b200_server_create.argtypes = [C.POINTER(ServerConfig)]
        L.hpgl_b200_server_submit.restype = C.c_longlong
        L.hpgl_b200_server_submit.argtypes = [C.c_void_p, C.POINTER(N.Job), C.POINTER(N.Result)]
        L.hpgl_b200_server_wait.restype = C.c_int
        L.hpgl_b200_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_int]
        L.hpgl_b200_server_stats.restype = C.c_int
        L.hpgl_b200_server_stats.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        L.hpgl_b200_server_destroy.restype = None
        L.hpgl_b200_server_destroy.argtypes = [C.c_void_p]
        L._server_bound = True
    return L


class Server:
    def __init__(self, hbm_budget_bytes=120 << 30, max_inflight=8, worker_threads=0):
        self.L = _bind()
        cfg = ServerConfig(hbm_budget_bytes, max_inflight, worker_threads)
        self.h = self.L.hpgl_b200_server_create(C.byref(cfg))
        if not self.h:
            code, msg = N.last_error()
            raise N.HpglError(code, msg)
        self.pending = {}

    def submit(self, job, precision=None, kind=None, dumps=False):
        p = N._Prepared(job, precision, kind, dumps, False, None)
        t = self.L.hpgl_b200_server_submit(self.h, C.byref(p.job), C.byref(p.result))
        if t < 0:
            code, msg = N.last_error()
            raise N.HpglError(code, msg)
        self.pending[t] = p
        return t

    def wait(self, ticket, timeout_ms=-1):
        """HPGL code of a finished job, or -1 while it runs."""
        return self.L.hpgl_b200_server_wait(self.h, ticket, timeout_ms)

    def result(self, ticket):
        code = self.wait(ticket)
        p = self.pending.pop(ticket)
        if code != 0:
            raise N.HpglError(code, N.last_error()[1])
        return p.collect()

    def stats(self):
        st = ServerStats()
        self.L.hpgl_b200_server_stats(self.h, C.byref(st))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def close(self):
        if self.h:
            self.L.hpgl_b200_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_stream(stream, precision="mixed", hbm_budget_bytes=120 << 30, max_inflight=8, keep_results=False):
    """Replay (arrival_s, job) pairs in real time; returns (stats, results)."""
    results = []
    with Server(hbm_budget_bytes, max_inflight) as srv:
        t0 = time.perf_counter()
        tickets = []
        for arrival, job in stream:
            delay = arrival - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets.append(srv.submit(job, precision=precision))
        for t in tickets:
            r = srv.result(t)
            if keep_results:
                results.append(r)
        st = srv.stats()
    return st, results
