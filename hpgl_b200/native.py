"""ctypes binding of the library's own entry points (include/hpgl.h).

``krige(job, ...)`` runs one job dict (the layout of ``hpgl_b200.workloads``)
through ``hpgl_b200_krige`` and returns numpy arrays; ``bench(job, ...)``
times the device-resident pipeline through ``hpgl_b200_bench``.  The library
is loaded from this package directory; a missing library is an error (there
is no fallback implementation).
"""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "hpgl.so")

KINDS = {"ok": 0, "sk": 1, "lvm": 2, "ik": 3, "median_ik": 4, "cok1": 5, "cok2": 6}
CONT_KINDS = ("ok", "sk", "lvm", "cok1", "cok2")
PRECISION = {"fp64": 0, "mixed": 1}

HPGL_OK = 0
HPGL_E_INVALID = 1
HPGL_E_CUDA = 2
HPGL_E_UNSUPPORTED = 3
HPGL_E_CAPACITY = 4
HPGL_E_INTERNAL = 5


class HpglShape(C.Structure):
    _fields_ = [("data", C.c_int * 3), ("strides", C.c_int * 3)]


class HpglIkParams(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3),
                ("max_neighbours", C.c_int), ("marginal_prob", C.c_double)]


class Job(C.Structure):
    _fields_ = [("kind", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("values", C.POINTER(C.c_float)), ("codes", C.POINTER(C.c_ubyte)),
                ("mask", C.POINTER(C.c_ubyte)), ("mean", C.POINTER(C.c_float)),
                ("params", C.POINTER(HpglIkParams)), ("n_params", C.c_int),
                ("sk_automatic_mean", C.c_int), ("sk_mean", C.c_double), ("median_marginal1", C.c_double),
                ("precision", C.c_int),
                ("secondary_values", C.POINTER(C.c_float)), ("secondary_mask", C.POINTER(C.c_ubyte)),
                ("primary_mean", C.c_double), ("secondary_mean", C.c_double), ("secondary_variance", C.c_double),
                ("correlation", C.c_double), ("secondary_cov", C.c_void_p),
                ("sequential", C.c_int), ("seed", C.c_longlong), ("simulation_mask", C.POINTER(C.c_ubyte)),
                ("category_means", C.POINTER(C.POINTER(C.c_float))), ("correlogram", C.c_int)]


class Result(C.Structure):
    _fields_ = [("out_values", C.POINTER(C.c_float)), ("out_codes", C.POINTER(C.c_ubyte)),
                ("out_mask", C.POINTER(C.c_ubyte)), ("variance", C.POINTER(C.c_double)),
                ("status", C.POINTER(C.c_byte)), ("nb_count", C.POINTER(C.c_int)),
                ("nb_index", C.POINTER(C.c_int)), ("weights", C.POINTER(C.c_double)),
                ("probs", C.POINTER(C.c_float)), ("nb_stride", C.c_int),
                ("systems", C.c_longlong), ("systems_fp64", C.c_longlong), ("failures", C.c_longlong),
                ("ms_plan", C.c_double), ("ms_h2d", C.c_double), ("ms_device", C.c_double),
                ("ms_d2h", C.c_double), ("ms_total", C.c_double), ("rounds", C.c_longlong)]


class Bench(C.Structure):
    _fields_ = [("iters", C.c_int), ("warmup", C.c_int), ("flush_bytes", C.c_longlong),
                ("ms_per_iter", C.POINTER(C.c_double)), ("ms_top_kernel", C.c_double),
                ("top_kernel", C.c_char * 64), ("launches_per_iter", C.c_int),
                ("systems", C.c_longlong), ("systems_fp64", C.c_longlong), ("ms_plan", C.c_double),
                ("ms_search", C.c_double), ("ms_resolve", C.c_double)]


_lib = None


class HpglError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("hpgl error %d: %s" % (code, message))
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("hpgl_b200/hpgl.so is not built (run python -m hpgl_b200.build)")
        _lib = C.CDLL(LIB_PATH)
        _lib.hpgl_get_last_exception_message.restype = C.c_char_p
        _lib.hpgl_b200_krige.restype = C.c_int
        _lib.hpgl_b200_krige.argtypes = [C.POINTER(Job), C.POINTER(Result)]
        _lib.hpgl_b200_bench.restype = C.c_int
        _lib.hpgl_b200_bench.argtypes = [C.POINTER(Job), C.POINTER(Result), C.POINTER(Bench)]
        _lib.hpgl_b200_version.restype = C.c_char_p
    return _lib


def last_error():
    L = lib()
    return L.hpgl_get_last_error(), L.hpgl_get_last_exception_message().decode()


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def make_params(plist):
    arr = (HpglIkParams * len(plist))()
    for i, p in enumerate(plist):
        q = arr[i]
        q.covariance_type = p["cov_type"]
        q.ranges[:] = p["ranges"]
        q.angles[:] = p["angles"]
        q.sill = p["sill"]
        q.nugget = p["nugget"]
        q.radiuses[:] = p["radii"]
        q.max_neighbours = p["max_neighbours"]
        q.marginal_prob = p.get("marginal_prob", 0.0)
    return arr


class _Prepared:
    """Holds the numpy arrays and ctypes structs of one call alive."""

    def __init__(self, job, precision, kind, dumps, sk_auto_mean, median_marginal1):
        self.kind = kind or job["kind"]
        nx, ny, nz = job["shape"]
        self.size = nx * ny * nz
        self.cont = self.kind in CONT_KINDS
        self.cok = self.kind in ("cok1", "cok2")
        self.params = job["params"] if self.kind == "ik" else job["params"][:1]
        self.K = len(self.params) if self.kind == "ik" else 1
        self.pk = make_params(self.params)
        self.values = np.ascontiguousarray(job["values"], dtype=np.float32) if self.cont else None
        self.codes = None if self.cont else np.ascontiguousarray(job["codes"], dtype=np.uint8)
        self.mask = np.ascontiguousarray(job["mask"], dtype=np.uint8)
        self.mean = np.ascontiguousarray(job["mean"], dtype=np.float32) if self.kind == "lvm" else None
        j = Job()
        j.kind = KINDS[self.kind]
        j.nx, j.ny, j.nz = nx, ny, nz
        j.values = _ptr(self.values, C.c_float)
        j.codes = _ptr(self.codes, C.c_ubyte)
        j.mask = _ptr(self.mask, C.c_ubyte)
        j.mean = _ptr(self.mean, C.c_float)
        j.params = C.cast(self.pk, C.POINTER(HpglIkParams))
        j.n_params = len(self.params)
        j.sk_automatic_mean = int(sk_auto_mean)
        j.sk_mean = job.get("sk_mean", 0.0)
        m1 = job.get("median_marginal1", 0.5) if median_marginal1 is None else median_marginal1
        j.median_marginal1 = m1
        j.precision = -1 if precision is None else PRECISION.get(precision, precision)
        if self.cok:
            self.svalues = np.ascontiguousarray(job["secondary_values"], dtype=np.float32)
            self.smask = np.ascontiguousarray(job["secondary_mask"], dtype=np.uint8)
            j.secondary_values = _ptr(self.svalues, C.c_float)
            j.secondary_mask = _ptr(self.smask, C.c_ubyte)
            j.primary_mean = job["primary_mean"]
            j.secondary_mean = job["secondary_mean"]
            j.secondary_variance = job.get("secondary_variance", 0.0)
            j.correlation = job["correlation"]
            if self.kind == "cok2":
                self.scov = cov_struct(job["secondary_cov"])
                j.secondary_cov = C.cast(C.pointer(self.scov), C.c_void_p)
        if job.get("sequential"):
            j.sequential = 1
            j.seed = int(job.get("seed", 0))
            sm = job.get("simulation_mask")
            self.sim_mask = None if sm is None else np.ascontiguousarray(sm, dtype=np.uint8)
            j.simulation_mask = _ptr(self.sim_mask, C.c_ubyte)
            cm = job.get("category_means")
            if cm is not None:
                self.cat_means = [np.ascontiguousarray(a, dtype=np.float32) for a in cm]
                self.cat_ptrs = (C.POINTER(C.c_float) * len(self.cat_means))(
                    *[_ptr(a, C.c_float) for a in self.cat_means])
                j.category_means = C.cast(self.cat_ptrs, C.POINTER(C.POINTER(C.c_float)))
                j.correlogram = int(bool(job.get("correlogram", False)))
        self.job = j
        self.out = self.values.copy() if self.cont else self.codes.copy()
        self.out_mask = self.mask.copy()
        # list stride; cokriging weights hold one more (the secondary's)
        cap = max(p["max_neighbours"] for p in self.params) + (1 if self.cok else 0)
        per_cat = self.kind == "ik" and any(
            (p["cov_type"], tuple(p["ranges"]), tuple(p["angles"]), p["sill"], p["nugget"], tuple(p["radii"]),
             p["max_neighbours"]) != (self.params[0]["cov_type"], tuple(self.params[0]["ranges"]),
                                      tuple(self.params[0]["angles"]), self.params[0]["sill"],
                                      self.params[0]["nugget"], tuple(self.params[0]["radii"]),
                                      self.params[0]["max_neighbours"]) for p in self.params)
        slots = self.size * (self.K if per_cat else 1)
        self.slots = slots
        self.cap = cap
        self.arrays = {}
        r = Result()
        r.out_values = _ptr(self.out, C.c_float) if self.cont else None
        r.out_codes = None if self.cont else _ptr(self.out, C.c_ubyte)
        r.out_mask = _ptr(self.out_mask, C.c_ubyte)
        if dumps:
            # dumps="variance": per-slot variance and status only (whole-grid
            # checks of large jobs); any other true value adds the neighbour
            # lists and weights
            a = self.arrays
            a["variance"] = np.full(slots, np.nan)
            a["status"] = np.full(slots, -2, dtype=np.int8)
            r.variance = _ptr(a["variance"], C.c_double)
            r.status = _ptr(a["status"], C.c_byte)
            if dumps != "variance":
                a["nb_count"] = np.full(slots, -1, dtype=np.int32)
                a["nb_index"] = np.full(slots * cap, -1, dtype=np.int32)
                a["weights"] = np.zeros(slots * cap)
                r.nb_count = _ptr(a["nb_count"], C.c_int)
                r.nb_index = _ptr(a["nb_index"], C.c_int)
                r.weights = _ptr(a["weights"], C.c_double)
        if not self.cont:
            self.arrays["probs"] = np.zeros(self.size * (self.K if self.kind == "ik" else 1), dtype=np.float32)
            r.probs = _ptr(self.arrays["probs"], C.c_float)
        r.nb_stride = cap
        self.result = r

    def collect(self):
        r = self.result
        out = dict(self.arrays)
        out["out"] = self.out
        out["out_mask"] = self.out_mask
        out["cap"] = self.cap
        for k in ("systems", "systems_fp64", "ms_plan", "ms_h2d", "ms_device", "ms_d2h", "ms_total", "rounds"):
            out[k] = getattr(r, k)
        return out


def krige(job, precision=None, kind=None, dumps=False, sk_auto_mean=False, median_marginal1=None):
    """Run one job on the GPU; returns a dict like oracle.run()."""
    L = lib()
    p = _Prepared(job, precision, kind, dumps, sk_auto_mean, median_marginal1)
    rc = L.hpgl_b200_krige(C.byref(p.job), C.byref(p.result))
    if rc != 0:
        raise HpglError(rc, L.hpgl_get_last_exception_message().decode())
    return p.collect()


def simulate(job, seed, kind=None, simulation_mask=None):
    """Sequential Gaussian simulation of a cont job (kind "sk": mean 0, "ok",
    or "lvm"); returns the dict of krige() with the simulated property."""
    j = dict(job, sequential=True, seed=seed, simulation_mask=simulation_mask)
    return krige(j, precision="fp64", kind=kind)


def simulate_indicator(job, seed, simulation_mask=None, category_means=None, correlogram=False):
    """Sequential indicator simulation of an IK job (codes, mask, one params
    entry per category with marginal_prob); `category_means`: optional mean
    cubes per category (with the correlogram weights when asked)."""
    j = dict(job, sequential=True, seed=seed, simulation_mask=simulation_mask, category_means=category_means,
             correlogram=correlogram)
    return krige(j, precision="fp64", kind="ik")


def bench(job, precision="mixed", iters=5, warmup=3, flush_bytes=256 << 20, kind=None):
    """Device-resident timing; returns (per-iteration ms array, info dict)."""
    L = lib()
    p = _Prepared(job, precision, kind, False, False, None)
    ms = np.zeros(iters)
    b = Bench()
    b.iters = iters
    b.warmup = warmup
    b.flush_bytes = flush_bytes
    b.ms_per_iter = _ptr(ms, C.c_double)
    rc = L.hpgl_b200_bench(C.byref(p.job), C.byref(p.result), C.byref(b))
    if rc != 0:
        raise HpglError(rc, L.hpgl_get_last_exception_message().decode())
    info = dict(ms_top_kernel=b.ms_top_kernel, top_kernel=b.top_kernel.decode(), launches=b.launches_per_iter,
                ms_search=b.ms_search, ms_resolve=b.ms_resolve,
                systems=b.systems, systems_fp64=b.systems_fp64, ms_plan=b.ms_plan, out=p.out,
                out_mask=p.out_mask)
    return ms, info


TUNE_MAX = 16


class Tune(C.Structure):
    _fields_ = [("candidates", C.c_int), ("schedule", C.c_int * TUNE_MAX), ("blocks_per_sm", C.c_int * TUNE_MAX),
                ("ms", C.c_double * TUNE_MAX), ("chosen", C.c_int), ("family", C.c_int), ("precision", C.c_int)]


def autotune(job, precision="mixed", kind=None):
    """Runs hpgl_b200_autotune on the job; returns the candidates tried and
    the launch setting now in force for its family and precision."""
    L = lib()
    p = _Prepared(job, precision, kind, False, False, None)
    t = Tune()
    rc = L.hpgl_b200_autotune(C.byref(p.job), C.byref(t))
    if rc != 0:
        raise HpglError(rc, L.hpgl_get_last_exception_message().decode())
    names = {0: "split", 1: "fused"}
    cands = [dict(schedule=names[t.schedule[i]], blocks_per_sm=t.blocks_per_sm[i], ms=t.ms[i])
             for i in range(t.candidates)]
    return dict(candidates=cands, chosen=cands[t.chosen], family=t.family, precision=t.precision)


def fma_peak(precision="mixed"):
    """Measured rate (TFLOP/s) of the CUDA-core pipe a precision solves on:
    "mixed" the FP32 pipe (packed multiply-adds), "fp64" the FP64 pipe
    (hpgl_b200_fma_peak)."""
    L = lib()
    v = C.c_double(0.0)
    rc = L.hpgl_b200_fma_peak({"fp64": 0, "mixed": 1}[precision], C.byref(v))
    if rc != 0:
        raise HpglError(rc, L.hpgl_get_last_exception_message().decode())
    return v.value


def set_launch(family, precision, schedule, blocks_per_sm=0):
    """Pins the launch setting of a family (0: <= 32 neighbours, 1: above)
    and precision ("fp64"/"mixed"): schedule "split" or "fused"."""
    L = lib()
    prec = {"fp64": 0, "mixed": 1}[precision]
    rc = L.hpgl_b200_set_launch(int(family), prec, {"split": 0, "fused": 1}[schedule], int(blocks_per_sm))
    if rc != 0:
        raise HpglError(rc, L.hpgl_get_last_exception_message().decode())


class HpglCovParams(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double)]


def cov_struct(p):
    cp = HpglCovParams()
    cp.covariance_type = p["cov_type"]
    cp.ranges[:] = p["ranges"]
    cp.angles[:] = p["angles"]
    cp.sill = p["sill"]
    cp.nugget = p["nugget"]
    return cp


def sk_weights(center, xs, ys, zs, p, entry="hpgl_simple_kriging_weights"):
    """Simple-kriging weights of one point through the C ABI entry `entry`
    (the reference's signature).  Returns float32 weights; raises HpglError."""
    L = lib()
    fn = getattr(L, entry)
    n = len(xs)
    c = (C.c_float * 3)(*[float(v) for v in center])
    x = np.ascontiguousarray(xs, dtype=np.float32)
    y = np.ascontiguousarray(ys, dtype=np.float32)
    z = np.ascontiguousarray(zs, dtype=np.float32)
    w = np.zeros(n, dtype=np.float32)
    cp = cov_struct(p)
    rc = fn(c, _ptr(x, C.c_float), _ptr(y, C.c_float), _ptr(z, C.c_float), n, C.byref(cp), _ptr(w, C.c_float))
    if rc != 0:
        code, msg = last_error()
        raise HpglError(code, msg)
    return w
