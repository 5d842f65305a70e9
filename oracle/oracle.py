"""ORACLE — test infrastructure only.

Python access to the two CPU checkers of the kriging path:

* ``restated``: oracle/hpgl_oracle.cpp, this repository's CPU restatement
  of the reference algorithm (built by oracle/build_oracle.sh);
* ``reference``: the reference's own kriging sources compiled by
  oracle/build_ref.sh into oracle/_ref/libhpgl_ref.so (present only where
  the reference checkout was available when it was built), reached through
  the reference's C ABI (api.h:218-277) and a dump driver.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module.
"""

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libhpgl_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhpgl_ref.so")

KINDS = {"ok": 0, "sk": 1, "lvm": 2, "ik": 3, "median_ik": 4}


class OracleParams(C.Structure):
    _fields_ = [("cov_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radii", C.c_int * 3),
                ("max_neighbours", C.c_int), ("marginal_prob", C.c_double)]


class HpglShape(C.Structure):
    _fields_ = [("data", C.c_int * 3), ("strides", C.c_int * 3)]


class HpglOkParams(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3),
                ("max_neighbours", C.c_int)]


class HpglSkParams(C.Structure):
    _fields_ = HpglOkParams._fields_ + [("automatic_mean", C.c_ubyte), ("mean", C.c_double)]


class HpglIkParams(C.Structure):
    _fields_ = HpglOkParams._fields_ + [("marginal_prob", C.c_double)]


class HpglMedianIkParams(C.Structure):
    _fields_ = HpglOkParams._fields_ + [("marginal_probs", C.c_double * 2)]


class HpglContArray(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("mask", C.POINTER(C.c_ubyte)), ("shape", HpglShape)]


class HpglIndArray(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_ubyte)), ("mask", C.POINTER(C.c_ubyte)), ("shape", HpglShape),
                ("indicator_count", C.c_int)]


_lib = None
_ref = None


def build_restated():
    subprocess.run(["bash", os.path.join(HERE, "build_oracle.sh")], check=True, capture_output=True)


def restated():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_restated()
        _lib = C.CDLL(ORACLE_SO)
        _lib.oracle_krige.restype = C.c_int
    return _lib


def reference_available():
    return os.path.exists(REF_SO)


def reference_src():
    """The reference checkout's src/ directory (read-only sources, test data
    and headers): $HPGL_REFERENCE_SRC, the same variable oracle/build_ref.sh
    reads, else the checkout's usual place.  Absent where only the prebuilt
    files travel."""
    return os.environ.get("HPGL_REFERENCE_SRC", "/root/reference/src")


_REF_OUTPUT = C.CFUNCTYPE(C.c_int, C.c_char_p, C.c_void_p)(lambda text, param: 0)
_REF_PROGRESS = C.CFUNCTYPE(C.c_int, C.c_char_p, C.c_int, C.c_void_p)(lambda stage, pct, param: 0)


def reference():
    global _ref
    if _ref is None:
        _ref = C.CDLL(REF_SO)
        _ref.hpgl_get_last_exception_message.restype = C.c_char_p
        _ref.ref_template.restype = C.c_int
        # the reference logs to stdout unless given handlers (output.cpp:9-20);
        # silence it so that a benchmark's JSON line stays alone on stdout
        _ref.hpgl_set_output_handler(_REF_OUTPUT, None)
        _ref.hpgl_set_progress_handler(_REF_PROGRESS, None)
    return _ref


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def oracle_params(p):
    o = OracleParams()
    o.cov_type = p["cov_type"]
    o.ranges[:] = p["ranges"]
    o.angles[:] = p["angles"]
    o.sill = p["sill"]
    o.nugget = p["nugget"]
    o.radii[:] = p["radii"]
    o.max_neighbours = p["max_neighbours"]
    o.marginal_prob = p.get("marginal_prob", 0.0)
    return o


def run(job, dumps=True, node_list=None, threads=0, sk_auto_mean=False, median_marginal1=None,
        kind=None):
    """Run the restated oracle on a job dict (see hpgl_b200.workloads).
    Returns a dict of numpy arrays: out (values or codes), out_mask and, with
    ``dumps``, per system slot: variance, status, nb_count, nb_index,
    weights, probs, via_template."""
    lib = restated()
    kind = kind or job["kind"]
    nx, ny, nz = job["shape"]
    size = nx * ny * nz
    params = job["params"]
    K = len(params) if kind == "ik" else 1
    parr = (OracleParams * K)(*[oracle_params(p) for p in params[:K]])
    cont = kind in ("ok", "sk", "lvm")
    values = np.ascontiguousarray(job["values"], dtype=np.float32) if cont else None
    codes = None if cont else np.ascontiguousarray(job["codes"], dtype=np.uint8)
    mask = np.ascontiguousarray(job["mask"], dtype=np.uint8)
    mean = np.ascontiguousarray(job["mean"], dtype=np.float32) if kind == "lvm" else None
    out = (values.copy() if cont else codes.copy())
    out_mask = mask.copy()
    slots = size * K
    cap = max(p["max_neighbours"] for p in params[:K])
    res = {}
    if dumps:
        res["variance"] = np.full(slots, np.nan)
        res["status"] = np.full(slots, -2, dtype=np.int8)
        res["nb_count"] = np.full(slots, -1, dtype=np.int32)
        res["nb_index"] = np.full(slots * cap, -1, dtype=np.int32)
        res["weights"] = np.zeros(slots * cap)
        res["probs"] = np.zeros(slots, dtype=np.float32)
        res["via_template"] = np.zeros(slots, dtype=np.uint8)
    nl = None if node_list is None else np.ascontiguousarray(node_list, dtype=np.int32)
    err = C.create_string_buffer(512)
    if median_marginal1 is None:
        median_marginal1 = job.get("median_marginal1", 0.5)
    rc = lib.oracle_krige(
        KINDS[kind], nx, ny, nz, _ptr(values, C.c_float), _ptr(codes, C.c_ubyte), _ptr(mask, C.c_ubyte),
        _ptr(mean, C.c_float), parr, K, C.c_double(job.get("sk_mean", 0.0)), int(sk_auto_mean),
        C.c_double(median_marginal1),
        _ptr(out, C.c_float) if cont else None, None if cont else _ptr(out, C.c_ubyte), _ptr(out_mask, C.c_ubyte),
        _ptr(res.get("variance"), C.c_double), _ptr(res.get("status"), C.c_byte),
        _ptr(res.get("nb_count"), C.c_int), _ptr(res.get("nb_index"), C.c_int),
        _ptr(res.get("weights"), C.c_double), _ptr(res.get("probs"), C.c_float),
        _ptr(res.get("via_template"), C.c_ubyte), cap, _ptr(nl, C.c_int), 0 if nl is None else len(nl),
        threads, err, 512)
    if rc != 0:
        raise RuntimeError("oracle: " + err.value.decode())
    res["out"] = out
    res["out_mask"] = out_mask
    res["cap"] = cap
    return res


def template(p, truncated=False):
    lib = restated()
    cap = (2 * p["radii"][0] + 1) * (2 * p["radii"][1] + 1) * (2 * p["radii"][2] + 1)
    buf = np.zeros(cap * 3, dtype=np.int32)
    n = lib.oracle_template(C.byref(oracle_params(p)), int(truncated), _ptr(buf, C.c_int), cap)
    return buf[: 3 * n].reshape(n, 3)


# ---- the reference itself (oracle/_ref) ------------------------------------

def _shape(shape):
    s = HpglShape()
    s.data[:] = shape
    s.strides[:] = (1, shape[0], shape[0] * shape[1])
    return s


def _ok_params(p, cls=HpglOkParams):
    o = cls()
    o.covariance_type = p["cov_type"]
    o.ranges[:] = p["ranges"]
    o.angles[:] = p["angles"]
    o.sill = p["sill"]
    o.nugget = p["nugget"]
    o.radiuses[:] = p["radii"]
    o.max_neighbours = p["max_neighbours"]
    return o


def ref_run(job, threads=0, kind=None, sk_auto_mean=False, median_marginal1=None):
    """Run the compiled reference through its own C ABI; returns (out, mask)
    starting, like geo.py does, from a clone of the input."""
    ref = reference()
    if threads > 0:
        ref.hpgl_set_thread_num(int(threads))
    kind = kind or job["kind"]
    shape = job["shape"]
    sh = _shape(shape)
    p0 = job["params"][0]
    mask = np.array(job["mask"], dtype=np.uint8)
    if kind in ("ok", "sk", "lvm"):
        values = np.array(job["values"], dtype=np.float32)
        out, out_mask = values.copy(), mask.copy()
        if kind == "ok":
            a = HpglContArray(_ptr(values, C.c_float), _ptr(mask, C.c_ubyte), sh)
            b = HpglContArray(_ptr(out, C.c_float), _ptr(out_mask, C.c_ubyte), sh)
            ref.hpgl_ordinary_kriging(C.byref(a), C.byref(_ok_params(p0)), C.byref(b))
        elif kind == "sk":
            sp = _ok_params(p0, HpglSkParams)
            sp.automatic_mean = int(sk_auto_mean)
            sp.mean = job.get("sk_mean", 0.0)
            ref.hpgl_simple_kriging(_ptr(values, C.c_float), _ptr(mask, C.c_ubyte), C.byref(sh), C.byref(sp),
                                    _ptr(out, C.c_float), _ptr(out_mask, C.c_ubyte), C.byref(sh))
        else:
            mean = np.array(job["mean"], dtype=np.float32)
            ref.hpgl_lvm_kriging(_ptr(values, C.c_float), _ptr(mask, C.c_ubyte), C.byref(sh),
                                 _ptr(mean, C.c_float), C.byref(sh), C.byref(_ok_params(p0)),
                                 _ptr(out, C.c_float), _ptr(out_mask, C.c_ubyte), C.byref(sh))
        return out, out_mask
    codes = np.array(job["codes"], dtype=np.uint8)
    out, out_mask = codes.copy(), mask.copy()
    K = len(job["params"])
    if kind == "ik":
        a = HpglIndArray(_ptr(codes, C.c_ubyte), _ptr(mask, C.c_ubyte), sh, K)
        b = HpglIndArray(_ptr(out, C.c_ubyte), _ptr(out_mask, C.c_ubyte), sh, K)
        ps = (HpglIkParams * K)()
        for k, p in enumerate(job["params"]):
            q = _ok_params(p, HpglIkParams)
            q.marginal_prob = p["marginal_prob"]
            ps[k] = q
        ref.hpgl_indicator_kriging(C.byref(a), C.byref(b), ps, K)
    else:
        a = HpglIndArray(_ptr(codes, C.c_ubyte), _ptr(mask, C.c_ubyte), sh, 2)
        b = HpglIndArray(_ptr(out, C.c_ubyte), _ptr(out_mask, C.c_ubyte), sh, 2)
        q = _ok_params(p0, HpglMedianIkParams)
        m1 = job.get("median_marginal1", 0.5) if median_marginal1 is None else median_marginal1
        q.marginal_probs[:] = (1.0 - m1, m1)
        ref.hpgl_median_ik(C.byref(a), C.byref(q), C.byref(b))
    return out, out_mask


class RefSimpleKriging:
    """The reference's stock simple-kriging entry point, hpgl_simple_kriging
    (api.cpp:261-288 -> simple_kriging.cpp:40-70 -> cont_kriging.h:75-113,
    per-node progress tick included), on a whole job with `threads` OpenMP
    threads (hpgl_set_thread_num).  The buffers are prepared once, as geo.py
    does (the output a clone of the input); ``call()`` is the C call alone.
    Every uninformed node is rewritten by each call (SK writes the mean where
    a system fails), so calls can repeat on the same buffers."""

    def __init__(self, job, threads):
        self.ref = reference()
        self.ref.hpgl_set_thread_num(int(threads))
        self.threads = int(self.ref.hpgl_get_thread_num())
        self.sh = _shape(job["shape"])
        self.values = np.array(job["values"], dtype=np.float32)
        self.mask = np.array(job["mask"], dtype=np.uint8)
        self.out, self.out_mask = self.values.copy(), self.mask.copy()
        self.sp = _ok_params(job["params"][0], HpglSkParams)
        self.sp.automatic_mean = 0
        self.sp.mean = job.get("sk_mean", 0.0)

    def call(self):
        self.ref.hpgl_simple_kriging(_ptr(self.values, C.c_float), _ptr(self.mask, C.c_ubyte), C.byref(self.sh),
                                     C.byref(self.sp), _ptr(self.out, C.c_float), _ptr(self.out_mask, C.c_ubyte),
                                     C.byref(self.sh))


def ref_dump(job, kind=None, category=0, marginal=None, threads=0):
    """Per-node dumps from the reference's own classes (oracle/ref_dump.cpp)."""
    ref = reference()
    kind = kind or job["kind"]
    nx, ny, nz = job["shape"]
    size = nx * ny * nz
    p = job["params"][category if kind == "ik" else 0]
    cap = p["max_neighbours"]
    res = dict(nb_count=np.full(size, -1, dtype=np.int32), nb_index=np.full(size * cap, -1, dtype=np.int32),
               weights=np.zeros(size * cap), variance=np.full(size, np.nan),
               status=np.full(size, -2, dtype=np.int32), estimate=np.full(size, np.nan))
    args = [_ptr(res["nb_count"], C.c_int), _ptr(res["nb_index"], C.c_int), _ptr(res["weights"], C.c_double),
            _ptr(res["variance"], C.c_double), _ptr(res["status"], C.c_int), _ptr(res["estimate"], C.c_double),
            int(threads)]
    mask = np.array(job["mask"], dtype=np.uint8)
    if kind in ("ok", "sk", "lvm"):
        values = np.array(job["values"], dtype=np.float32)
        mean = np.array(job["mean"], dtype=np.float32) if kind == "lvm" else None
        rc = ref.ref_dump_cont(KINDS[kind], nx, ny, nz, _ptr(values, C.c_float), _ptr(mask, C.c_ubyte),
                               _ptr(mean, C.c_float), C.byref(_ok_params(p)), C.c_double(job.get("sk_mean", 0.0)),
                               cap, *args)
    else:
        codes = np.array(job["codes"], dtype=np.uint8)
        if marginal is None:
            marginal = p["marginal_prob"] if kind == "ik" else job.get("median_marginal1", 0.5)
        rc = ref.ref_dump_ind(KINDS[kind], nx, ny, nz, _ptr(codes, C.c_ubyte), _ptr(mask, C.c_ubyte),
                              int(category), C.byref(_ok_params(p)), C.c_double(marginal), cap, *args)
    if rc != 0:
        raise RuntimeError("reference dump failed")
    res["cap"] = cap
    return res


def ref_template(p):
    ref = reference()
    cap = (2 * p["radii"][0] + 1) * (2 * p["radii"][1] + 1) * (2 * p["radii"][2] + 1)
    buf = np.zeros(cap * 3, dtype=np.int32)
    n = ref.ref_template(C.byref(_ok_params(p)), _ptr(buf, C.c_int), cap)
    return buf[: 3 * n].reshape(n, 3)


def ref_sample(job, node_list, threads=0, kind=None):
    """The reference's own per-node kriging on `node_list` (OK or SK);
    returns the estimates (NaN where the system failed)."""
    ref = reference()
    kind = kind or job["kind"]
    nx, ny, nz = job["shape"]
    values = np.array(job["values"], dtype=np.float32)
    mask = np.array(job["mask"], dtype=np.uint8)
    nl = np.ascontiguousarray(node_list, dtype=np.int32)
    out = np.zeros(len(nl), dtype=np.float32)
    rc = ref.ref_sample_cont(KINDS[kind], nx, ny, nz, _ptr(values, C.c_float), _ptr(mask, C.c_ubyte),
                             C.byref(_ok_params(job["params"][0])), C.c_double(job.get("sk_mean", 0.0)),
                             _ptr(nl, C.c_int), len(nl), int(threads), _ptr(out, C.c_float))
    if rc != 0:
        raise RuntimeError("reference sample failed")
    return out


def sk_weights(center, xs, ys, zs, p):
    """Restated hpgl_simple_kriging_weights; returns (status, float32 weights)."""
    lib = restated()
    n = len(xs)
    c = np.ascontiguousarray(center, dtype=np.float32)
    x = np.ascontiguousarray(xs, dtype=np.float32)
    y = np.ascontiguousarray(ys, dtype=np.float32)
    z = np.ascontiguousarray(zs, dtype=np.float32)
    w = np.zeros(n, dtype=np.float32)
    rc = lib.oracle_sk_weights(_ptr(c, C.c_float), _ptr(x, C.c_float), _ptr(y, C.c_float), _ptr(z, C.c_float), n,
                               C.byref(oracle_params(p)), _ptr(w, C.c_float))
    return rc, w


def ref_sk_weights(center, xs, ys, zs, p):
    """The compiled reference's hpgl_simple_kriging_weights (float32 weights)."""
    ref = reference()

    class CovParams(C.Structure):
        _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                    ("sill", C.c_double), ("nugget", C.c_double)]
    cp = CovParams()
    cp.covariance_type = p["cov_type"]
    cp.ranges[:] = p["ranges"]
    cp.angles[:] = p["angles"]
    cp.sill = p["sill"]
    cp.nugget = p["nugget"]
    n = len(xs)
    c = (C.c_float * 3)(*center)
    x = np.ascontiguousarray(xs, dtype=np.float32)
    y = np.ascontiguousarray(ys, dtype=np.float32)
    z = np.ascontiguousarray(zs, dtype=np.float32)
    w = np.zeros(n, dtype=np.float32)
    ref.hpgl_simple_kriging_weights(c, _ptr(x, C.c_float), _ptr(y, C.c_float), _ptr(z, C.c_float), n, C.byref(cp),
                                    _ptr(w, C.c_float))
    return w


class HpglCovParams(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double)]


class HpglCokM1Params(C.Structure):
    _fields_ = HpglOkParams._fields_ + [("primary_mean", C.c_double), ("secondary_mean", C.c_double),
                                        ("secondary_variance", C.c_double), ("correlation_coef", C.c_double)]


class HpglCokM2Params(C.Structure):
    _fields_ = [("primary_cov", HpglCovParams), ("secondary_cov", HpglCovParams), ("radiuses", C.c_int * 3),
                ("max_neighbours", C.c_int), ("primary_mean", C.c_double), ("secondary_mean", C.c_double),
                ("correlation_coef", C.c_double)]


def _cov_params(p):
    cp = HpglCovParams()
    cp.covariance_type = p["cov_type"]
    cp.ranges[:] = p["ranges"]
    cp.angles[:] = p["angles"]
    cp.sill = p["sill"]
    cp.nugget = p["nugget"]
    return cp


def cokriging(job, dumps=True, node_list=None, threads=0):
    """Restated colocated simple cokriging (job kind "cok1" or "cok2", see
    hpgl_b200.workloads.cokriging_job).  Returns out, out_mask and, with
    ``dumps``, per node: status, nb_count, nb_index (cap per node), weights
    (cap + 1 per node)."""
    lib = restated()
    mark = {"cok1": 1, "cok2": 2}[job["kind"]]
    nx, ny, nz = job["shape"]
    size = nx * ny * nz
    p = job["params"][0]
    cap = p["max_neighbours"]
    values = np.ascontiguousarray(job["values"], dtype=np.float32)
    mask = np.ascontiguousarray(job["mask"], dtype=np.uint8)
    sv = np.ascontiguousarray(job["secondary_values"], dtype=np.float32)
    sm = np.ascontiguousarray(job["secondary_mask"], dtype=np.uint8)
    out, out_mask = values.copy(), mask.copy()
    res = {}
    if dumps:
        res["status"] = np.full(size, -2, dtype=np.int8)
        res["nb_count"] = np.full(size, -1, dtype=np.int32)
        res["nb_index"] = np.full(size * cap, -1, dtype=np.int32)
        res["weights"] = np.zeros(size * (cap + 1))
    sp = oracle_params(job["secondary_cov"]) if mark == 2 else None
    nl = None if node_list is None else np.ascontiguousarray(node_list, dtype=np.int32)
    err = C.create_string_buffer(512)
    rc = lib.oracle_cokriging(
        mark, nx, ny, nz, _ptr(values, C.c_float), _ptr(mask, C.c_ubyte), _ptr(sv, C.c_float), _ptr(sm, C.c_ubyte),
        C.byref(oracle_params(p)), None if sp is None else C.byref(sp), C.c_double(job["primary_mean"]),
        C.c_double(job["secondary_mean"]), C.c_double(job.get("secondary_variance", 0.0)),
        C.c_double(job["correlation"]), _ptr(out, C.c_float), _ptr(out_mask, C.c_ubyte),
        _ptr(res.get("status"), C.c_byte), _ptr(res.get("nb_count"), C.c_int), _ptr(res.get("nb_index"), C.c_int),
        _ptr(res.get("weights"), C.c_double), cap, _ptr(nl, C.c_int), 0 if nl is None else len(nl), threads, err, 512)
    if rc != 0:
        raise RuntimeError("oracle: " + err.value.decode())
    res["out"] = out
    res["out_mask"] = out_mask
    res["cap"] = cap
    return res


def ref_cokriging(job):
    """The compiled reference's hpgl_simple_cokriging_mark1/2 through its C
    ABI, from a clone of the primary input like geo.py; returns (out, mask)."""
    ref = reference()
    sh = _shape(job["shape"])
    p = job["params"][0]
    values = np.array(job["values"], dtype=np.float32)
    mask = np.array(job["mask"], dtype=np.uint8)
    sv = np.array(job["secondary_values"], dtype=np.float32)
    sm = np.array(job["secondary_mask"], dtype=np.uint8)
    out, out_mask = values.copy(), mask.copy()
    a = HpglContArray(_ptr(values, C.c_float), _ptr(mask, C.c_ubyte), sh)
    s = HpglContArray(_ptr(sv, C.c_float), _ptr(sm, C.c_ubyte), sh)
    b = HpglContArray(_ptr(out, C.c_float), _ptr(out_mask, C.c_ubyte), sh)
    if job["kind"] == "cok1":
        q = HpglCokM1Params()
        base = _ok_params(p)
        for name, _ in HpglOkParams._fields_:
            setattr(q, name, getattr(base, name))
        q.primary_mean = job["primary_mean"]
        q.secondary_mean = job["secondary_mean"]
        q.secondary_variance = job["secondary_variance"]
        q.correlation_coef = job["correlation"]
        ref.hpgl_simple_cokriging_mark1(C.byref(a), C.byref(s), C.byref(q), C.byref(b))
    else:
        q = HpglCokM2Params()
        q.primary_cov = _cov_params(p)
        q.secondary_cov = _cov_params(job["secondary_cov"])
        q.radiuses[:] = p["radii"]
        q.max_neighbours = p["max_neighbours"]
        q.primary_mean = job["primary_mean"]
        q.secondary_mean = job["secondary_mean"]
        q.correlation_coef = job["correlation"]
        ref.hpgl_simple_cokriging_mark2(C.byref(a), C.byref(s), C.byref(q), C.byref(b))
    return out, out_mask


# ---- INC / GSLIB property files -----------------------------------------------

class OracleIoError(RuntimeError):
    pass


def _b(s):
    return s if isinstance(s, bytes) else os.fsencode(s)


def read_inc(path, size, undefined, is_byte=False, values=()):
    """Restated reader (textio_oracle.cpp).  Returns (data, mask) of length
    `size`, or raises OracleIoError(message, partial data, partial mask)."""
    lib = restated()
    lib.oracle_read_inc.restype = C.c_int
    data = np.zeros(size, dtype=np.uint8 if is_byte else np.float32)
    mask = np.zeros(size, dtype=np.uint8)
    vals = np.ascontiguousarray(np.array(values, dtype=np.uint8).reshape(-1))
    err = C.create_string_buffer(1024)
    rc = lib.oracle_read_inc(_b(path), int(bool(is_byte)), C.c_float(0.0 if is_byte else undefined),
                             int(undefined) if is_byte else 0, C.c_longlong(size),
                             None if is_byte else _ptr(data, C.c_float), _ptr(data, C.c_ubyte) if is_byte else None,
                             _ptr(mask, C.c_ubyte), _ptr(vals, C.c_ubyte), len(vals), err, 1024)
    if rc != 0:
        e = OracleIoError(err.value.decode(errors="replace"))
        e.data, e.mask = data, mask
        raise e
    return data, mask


def inc_count(path):
    lib = restated()
    lib.oracle_inc_count.restype = C.c_longlong
    err = C.create_string_buffer(1024)
    n = lib.oracle_inc_count(_b(path), err, 1024)
    if n < 0:
        raise OracleIoError(err.value.decode(errors="replace"))
    return int(n)


def remap_table(values, indicator_count):
    """init_remap_table (api.cpp:117-136)."""
    values = list(values)
    if len(values) == indicator_count:
        return values
    if len(values) > indicator_count:
        return values[:indicator_count]
    return list(range(indicator_count))


def write_prop(path, name, data, mask, undefined, fmt="inc", is_byte=False, remap=()):
    """Restated writer; fmt "inc" or "gslib".  For bytes, `remap` is the
    table (remap_table's result) and `undefined` the byte written for
    uninformed cells."""
    lib = restated()
    lib.oracle_write_prop.restype = C.c_int
    data = np.ascontiguousarray(data, dtype=np.uint8 if is_byte else np.float32).reshape(-1)
    mask = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    rm = np.ascontiguousarray(np.array(remap, dtype=np.uint8).reshape(-1))
    err = C.create_string_buffer(1024)
    rc = lib.oracle_write_prop(0 if fmt == "inc" else 1, int(bool(is_byte)), _b(path), _b(name),
                               None if is_byte else _ptr(data, C.c_float), _ptr(data, C.c_ubyte) if is_byte else None,
                               _ptr(mask, C.c_ubyte), C.c_longlong(data.size),
                               C.c_float(0.0 if is_byte else undefined), C.c_ubyte(int(undefined) & 0xff if is_byte else 0),
                               _ptr(rm, C.c_ubyte), len(rm), err, 1024)
    if rc != 0:
        raise OracleIoError(err.value.decode(errors="replace"))


def ref_read_inc(path, size, undefined, is_byte=False, values=()):
    """The reference's own hpgl_read_inc_file_float/_byte.  Only for files it
    reads without an error: its exceptions cross the C boundary and end the
    process."""
    ref = reference()
    data = np.zeros(size, dtype=np.uint8 if is_byte else np.float32)
    mask = np.zeros(size, dtype=np.uint8)
    if is_byte:
        vals = np.ascontiguousarray(np.array(values, dtype=np.uint8).reshape(-1))
        ref.hpgl_read_inc_file_byte(_b(path), int(undefined), int(size), _ptr(data, C.c_ubyte),
                                    _ptr(mask, C.c_ubyte), _ptr(vals, C.c_ubyte), len(vals))
    else:
        ref.hpgl_read_inc_file_float(_b(path), C.c_float(undefined), int(size), _ptr(data, C.c_float),
                                     _ptr(mask, C.c_ubyte))
    return data, mask


def ref_write_prop(path, name, data, mask, undefined, fmt="inc", is_byte=False, values=(), indicator_count=None):
    """The reference's own writers (api.cpp:101-193), one-dimensional shape."""
    ref = reference()
    data = np.ascontiguousarray(data, dtype=np.uint8 if is_byte else np.float32).reshape(-1)
    mask = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    sh = _shape((data.size, 1, 1))
    if is_byte:
        vals = np.ascontiguousarray(np.array(values, dtype=np.uint8).reshape(-1))
        arr = HpglIndArray(_ptr(data, C.c_ubyte), _ptr(mask, C.c_ubyte), sh,
                           indicator_count if indicator_count is not None else len(vals))
        if fmt == "inc":
            ref.hpgl_write_inc_file_byte(_b(path), C.byref(arr), int(undefined), _b(name), _ptr(vals, C.c_ubyte),
                                         len(vals))
        else:
            ref.hpgl_write_gslib_byte_property(C.byref(arr), _b(path), _b(name), C.c_double(undefined),
                                               _ptr(vals, C.c_ubyte), len(vals))
    else:
        arr = HpglContArray(_ptr(data, C.c_float), _ptr(mask, C.c_ubyte), sh)
        if fmt == "inc":
            ref.hpgl_write_inc_file_float(_b(path), C.byref(arr), C.c_float(undefined), _b(name))
        else:
            ref.hpgl_write_gslib_cont_property(C.byref(arr), _b(path), _b(name), C.c_double(undefined))


# ---- experimental variograms (_cvariogram) ---------------------------------------

REF_CV_SO = os.path.join(HERE, "_ref", "libcvariogram_ref.so")


class CvVector(C.Structure):
    _fields_ = [("data", C.c_double * 3)]


class CvEllipsoid(C.Structure):
    _fields_ = [("direction1", CvVector), ("direction2", CvVector), ("direction3", CvVector), ("R1", C.c_double),
                ("R2", C.c_double), ("R3", C.c_double)]


class CvTemplate(C.Structure):
    _fields_ = [("lag_width", C.c_double), ("lag_separation", C.c_double), ("tol_distance", C.c_double),
                ("num_lags", C.c_int), ("first_lag_distance", C.c_double), ("ellipsoid", CvEllipsoid)]


class CvHardData(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("mask", C.POINTER(C.c_ubyte)), ("data_shape", C.c_int * 3),
                ("data_strides", C.c_int * 3), ("mask_shape", C.c_int * 3), ("mask_strides", C.c_int * 3)]


class CvPointSet(C.Structure):
    _fields_ = [("xs", C.POINTER(C.c_float)), ("ys", C.POINTER(C.c_float)), ("zs", C.POINTER(C.c_float)),
                ("values", C.POINTER(C.c_float)), ("size", C.c_int)]


class CvFloatData(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("shape", C.c_int * 3), ("strides", C.c_int * 3)]


_ref_cv = None


def reference_cv_available():
    return os.path.exists(REF_CV_SO)


def ref_cv():
    global _ref_cv
    if _ref_cv is None:
        _ref_cv = C.CDLL(REF_CV_SO)
        _ref_cv.ref_cvar_lag_areas.restype = C.c_longlong
    return _ref_cv


def cv_template(lag_width, lag_separation, tol_distance, num_lags, first_lag_distance, radii, angles):
    """A search template with the restated fill_ellipsoid_directions."""
    t = CvTemplate()
    t.lag_width, t.lag_separation, t.tol_distance = lag_width, lag_separation, tol_distance
    t.num_lags, t.first_lag_distance = num_lags, first_lag_distance
    d = (C.c_double * 9)()
    restated().oracle_fill_ellipsoid_directions(d, C.c_double(angles[0]), C.c_double(angles[1]),
                                                C.c_double(angles[2]))
    t.ellipsoid.direction1.data[:] = d[0:3]
    t.ellipsoid.direction2.data[:] = d[3:6]
    t.ellipsoid.direction3.data[:] = d[6:9]
    t.ellipsoid.R1, t.ellipsoid.R2, t.ellipsoid.R3 = radii
    return t


def cv_hard_data(data, mask):
    """(struct, keep-alive arrays) for a 3-D float32 property and uint8 mask
    of any memory order (strides in elements)."""
    data = np.asarray(data, dtype=np.float32)
    mask = np.asarray(mask, dtype=np.uint8)
    hd = CvHardData()
    hd.data = _ptr(data, C.c_float)
    hd.mask = _ptr(mask, C.c_ubyte)
    hd.data_shape[:] = data.shape
    hd.mask_shape[:] = mask.shape
    hd.data_strides[:] = [s // data.itemsize for s in data.strides]
    hd.mask_strides[:] = [s // mask.itemsize for s in mask.strides]
    return hd, (data, mask)


def variograms(templ, data, mask, percent=100, lags=None):
    """Restated calc_variograms: dict of result (float32), seq_sums, exact_sums, counts."""
    lib = restated()
    n = templ.num_lags if lags is None else lags
    hd, keep = cv_hard_data(data, mask)
    out = {"result": np.zeros(n, np.float32), "seq_sums": np.zeros(n), "exact_sums": np.zeros(n),
           "counts": np.zeros(n, np.int64)}
    lib.oracle_calc_variograms(C.byref(templ), C.byref(hd), _ptr(out["result"], C.c_float),
                               _ptr(out["seq_sums"], C.c_double), _ptr(out["exact_sums"], C.c_double),
                               _ptr(out["counts"], C.c_longlong), n, percent)
    return out


def cv_point_set(xs, ys, zs, values):
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (xs, ys, zs, values)]
    ps = CvPointSet(_ptr(arrs[0], C.c_float), _ptr(arrs[1], C.c_float), _ptr(arrs[2], C.c_float),
                    _ptr(arrs[3], C.c_float), len(arrs[3]))
    return ps, arrs


def variograms_points(templ, xs, ys, zs, values, lags=None):
    lib = restated()
    n = templ.num_lags if lags is None else lags
    ps, keep = cv_point_set(xs, ys, zs, values)
    out = {"result": np.zeros(n, np.float32), "seq_sums": np.zeros(n), "exact_sums": np.zeros(n),
           "counts": np.zeros(n, np.int64)}
    lib.oracle_calc_variograms_points(C.byref(templ), C.byref(ps), _ptr(out["result"], C.c_float),
                                      _ptr(out["seq_sums"], C.c_double), _ptr(out["exact_sums"], C.c_double),
                                      _ptr(out["counts"], C.c_longlong), n)
    return out


def ref_variograms(templ, data, mask, lags=None):
    """The reference's calc_variograms (percent 100)."""
    n = templ.num_lags if lags is None else lags
    hd, keep = cv_hard_data(data, mask)
    res = np.zeros(n, np.float32)
    ref_cv().calc_variograms(C.byref(templ), C.byref(hd), _ptr(res, C.c_float), n, 100)
    return res


def ref_variograms_points(templ, xs, ys, zs, values, lags=None):
    n = templ.num_lags if lags is None else lags
    ps, keep = cv_point_set(xs, ys, zs, values)
    res = np.zeros(n, np.float32)
    ref_cv().calc_variograms_from_point_set(C.byref(templ), C.byref(ps), _ptr(res, C.c_float), n)
    return res


def _float_data(a):
    fd = CvFloatData()
    fd.data = _ptr(a, C.c_float)
    fd.shape[:] = list(a.shape) + [1] * (3 - a.ndim)
    st = [s // a.itemsize for s in a.strides]
    fd.strides[:] = st + [0] * (3 - a.ndim)
    return fd


def stack_layers(layers, markers, nz, scalez, blank_value, result, reference=False):
    """stack_layers into `result` (3-D float32, modified in place)."""
    arr = (CvFloatData * len(layers))(*[_float_data(l) for l in layers])
    mk = (C.c_int * len(markers))(*markers)
    res = _float_data(result)
    if reference:
        ref_cv().cvar_stack_layers(arr, mk, len(layers), nz, C.c_float(scalez), blank_value, C.byref(res))
    else:
        restated().oracle_stack_layers(arr, mk, len(layers), nz, C.c_float(scalez), blank_value, C.byref(res))
    return result


# ---- sequential Gaussian simulation --------------------------------------------

class HpglSgsParams(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3), ("max_neighbours", C.c_int),
                ("kriging_kind", C.c_int), ("seed", C.c_long), ("min_neighbours", C.c_int)]


class HpglNonParametricCdf(C.Structure):
    _fields_ = [("values", C.POINTER(C.c_float)), ("probs", C.POINTER(C.c_float)), ("size", C.c_longlong)]


class HpglFloatArray(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("shape", HpglShape)]


class HpglUbyteArray(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_ubyte)), ("shape", HpglShape)]


def cdf_transform(values, cdf, direction, mask=None):
    """Normal-score transform of a float32 array through a (values, probs)
    CDF: direction 0 to the standard normal, 1 back (restated)."""
    cv = np.ascontiguousarray(cdf[0], dtype=np.float32)
    cp = np.ascontiguousarray(cdf[1], dtype=np.float32)
    out = np.array(values, dtype=np.float32)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    restated().oracle_cdf_transform(_ptr(out, C.c_float), _ptr(out, C.c_float), _ptr(m, C.c_ubyte),
                                    C.c_longlong(out.size), _ptr(cv, C.c_float), _ptr(cp, C.c_float),
                                    C.c_longlong(cv.size), int(direction))
    return out


def sgs(job, ordinary=False, seed=1, sim_mask=None, lvm=None, cdf=None):
    """Restated sequential Gaussian simulation: (values, mask, order of the
    simulated nodes).  `cdf` = (values, probs): the normal-score transforms
    around it (sequential_gaussian_simulation.cpp:32-35, 72-73, 97-103,
    119-123)."""
    lib = restated()
    nx, ny, nz = job["shape"]
    values = np.array(job["values"], dtype=np.float32)
    mask = np.array(job["mask"], dtype=np.uint8)
    if cdf is not None:
        values = cdf_transform(values, cdf, 0, mask)
        if lvm is not None:
            lvm = cdf_transform(lvm, cdf, 0)
    order = np.zeros(values.size, dtype=np.int32)
    n_order = C.c_int(0)
    sm = None if sim_mask is None else np.ascontiguousarray(sim_mask, dtype=np.uint8)
    lv = None if lvm is None else np.ascontiguousarray(lvm, dtype=np.float32)
    err = C.create_string_buffer(512)
    rc = lib.oracle_sgs(nx, ny, nz, _ptr(values, C.c_float), _ptr(mask, C.c_ubyte),
                        C.byref(oracle_params(job["params"][0])), int(ordinary), _ptr(lv, C.c_float),
                        C.c_longlong(seed), _ptr(sm, C.c_ubyte), _ptr(order, C.c_int), C.byref(n_order), err, 512)
    if rc != 0:
        raise RuntimeError("oracle: " + err.value.decode())
    if cdf is not None:
        values = cdf_transform(values, cdf, 1, mask)
    return values, mask, order[:n_order.value]


def sgs_draws(seed, n):
    """The standard normal quantiles of the first n draws (restated generator)."""
    xp = np.zeros(n)
    restated().oracle_sgs_draws(C.c_longlong(seed), C.c_longlong(n), _ptr(xp, C.c_double))
    return xp


def ref_sgs(job, ordinary=False, seed=1, sim_mask=None, lvm=None, cdf=None):
    """The reference's hpgl_sgs_simulation / hpgl_sgs_lvm_simulation, compiled
    with oracle/ref_shim's boost::mt11213b and the generated prime table;
    `cdf` = (values, probs) or None."""
    ref = reference()
    nx, ny, nz = job["shape"]
    sh = _shape((nx, ny, nz))
    values = np.array(job["values"], dtype=np.float32)
    mask = np.array(job["mask"], dtype=np.uint8)
    arr = HpglContArray(_ptr(values, C.c_float), _ptr(mask, C.c_ubyte), sh)
    p = job["params"][0]
    q = HpglSgsParams()
    q.covariance_type = p["cov_type"]
    q.ranges[:] = p["ranges"]
    q.angles[:] = p["angles"]
    q.sill, q.nugget = p["sill"], p["nugget"]
    q.radiuses[:] = p["radii"]
    q.max_neighbours = p["max_neighbours"]
    q.kriging_kind = 0 if ordinary else 1
    q.seed = seed
    q.min_neighbours = 0
    sm_keep = None
    smp = None
    if sim_mask is not None:
        sm_keep = np.ascontiguousarray(sim_mask, dtype=np.uint8)
        smp = C.byref(HpglUbyteArray(_ptr(sm_keep, C.c_ubyte), sh))
    cdfp = None
    if cdf is not None:
        cv = np.ascontiguousarray(cdf[0], dtype=np.float32)
        cp = np.ascontiguousarray(cdf[1], dtype=np.float32)
        cdfp = C.byref(HpglNonParametricCdf(_ptr(cv, C.c_float), _ptr(cp, C.c_float), cv.size))
    if lvm is not None:
        lv = np.ascontiguousarray(lvm, dtype=np.float32)
        fa = HpglFloatArray(_ptr(lv, C.c_float), sh)
        ref.hpgl_sgs_lvm_simulation(C.byref(arr), C.byref(q), cdfp, C.byref(fa), smp)
    else:
        ref.hpgl_sgs_simulation(C.byref(arr), C.byref(q), cdfp, None, smp)
    return values, mask


def _ik_param_array(params):
    arr = (OracleParams * len(params))()
    for i, p in enumerate(params):
        arr[i] = oracle_params(p)
    return arr


def sis(shape, codes, mask, params, seed=1, sim_mask=None, lvm=None, correlogram=False):
    """Restated sequential indicator simulation: (codes, mask).  `params`:
    one dict per category (with marginal_prob); `lvm`: K mean cubes."""
    nx, ny, nz = shape
    c = np.array(codes, dtype=np.uint8)
    m = np.array(mask, dtype=np.uint8)
    K = len(params)
    sm = None if sim_mask is None else np.ascontiguousarray(sim_mask, dtype=np.uint8)
    keep = []
    lv = None
    if lvm is not None:
        keep = [np.ascontiguousarray(a, dtype=np.float32) for a in lvm]
        lv = (C.POINTER(C.c_float) * K)(*[_ptr(a, C.c_float) for a in keep])
    err = C.create_string_buffer(512)
    rc = restated().oracle_sis(nx, ny, nz, _ptr(c, C.c_ubyte), _ptr(m, C.c_ubyte), _ik_param_array(params), K, lv,
                               int(correlogram), C.c_longlong(seed), _ptr(sm, C.c_ubyte), err, 512)
    if rc != 0:
        raise RuntimeError("oracle: " + err.value.decode())
    return c, m


class HpglIndMaskedArray(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_ubyte)), ("mask", C.POINTER(C.c_ubyte)), ("shape", HpglShape),
                ("indicator_count", C.c_int)]


class HpglIkParams(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3), ("max_neighbours", C.c_int),
                ("marginal_prob", C.c_double)]


def ik_params_array(params):
    arr = (HpglIkParams * len(params))()
    for i, p in enumerate(params):
        q = arr[i]
        q.covariance_type = p["cov_type"]
        q.ranges[:] = p["ranges"]
        q.angles[:] = p["angles"]
        q.sill, q.nugget = p["sill"], p["nugget"]
        q.radiuses[:] = p["radii"]
        q.max_neighbours = p["max_neighbours"]
        q.marginal_prob = p.get("marginal_prob", 0.0)
    return arr


def ref_sis(shape, codes, mask, params, seed=1, sim_mask=None, lvm=None, correlogram=False):
    """The reference's hpgl_sis_simulation / hpgl_sis_simulation_lvm."""
    ref = reference()
    sh = _shape(shape)
    c = np.array(codes, dtype=np.uint8)
    m = np.array(mask, dtype=np.uint8)
    K = len(params)
    arr = HpglIndMaskedArray(_ptr(c, C.c_ubyte), _ptr(m, C.c_ubyte), sh, K)
    sm_keep = None
    smp = None
    if sim_mask is not None:
        sm_keep = np.ascontiguousarray(sim_mask, dtype=np.uint8)
        smp = C.byref(HpglUbyteArray(_ptr(sm_keep, C.c_ubyte), sh))
    ps = ik_params_array(params)
    if lvm is not None:
        keep = [np.ascontiguousarray(a, dtype=np.float32) for a in lvm]
        fa = (HpglFloatArray * K)(*[HpglFloatArray(_ptr(a, C.c_float), sh) for a in keep])
        ref.hpgl_sis_simulation_lvm(C.byref(arr), ps, fa, K, int(seed), smp, int(correlogram))
    else:
        ref.hpgl_sis_simulation(C.byref(arr), ps, K, int(seed), smp)
    return c, m
