"""Kriging entry points with the names and arguments of the reference's
geo_bsd/geo.py (Python 2) — ``ordinary_kriging`` (geo.py:381-399),
``simple_kriging`` (:401-425), ``lvm_kriging`` (:427-450), ``median_ik``
(:452-469), ``indicator_kriging`` (:489-509), ``simple_cokriging_markI``
(:512-534), ``simple_cokriging_markII`` (:536-572), ``simple_kriging_weights``
(:568-600) — plus the property, grid and covariance classes they take
(:85-166), the thread/handler settings (:364-368, 602-618) and the INC /
GSLIB property files: ``write_property`` (:277-305), ``write_gslib_property``
(:307-322), ``load_cont_property`` (:324-329), ``read_inc_file_float``
(:331-342), ``read_inc_file_byte`` (:344-355), ``load_ind_property``
(:357-362), ``get_gslib_property`` (:608-616).

Differences from the reference, all additive:
* every call checks the library's last-error state and raises
  ``HpglError`` (the reference's C++ exceptions crossed the C boundary);
* each kriging call takes an optional ``precision`` keyword ("fp64" — the
  reference's arithmetic, bit for bit — or "mixed"); None uses the library
  default (``set_precision``);
* ``load_cont_property`` / ``load_ind_property`` without ``size`` read the
  file's values with the same INC rules as with a size (the count comes
  from ``hpgl_b200_inc_count_values``), where the reference switched to a
  pure-Python reader with looser rules; the result is one-dimensional, as
  the reference's was;
* ``write_property`` of an indicator property passes ``indicator_values``
  as bytes (the reference handed the bytes of an int64 array to a uint8
  pointer, so the table it wrote through held the low bytes of its first
  values' int64 words);
* file names and property names may be ``str`` (encoded with
  ``os.fsencode`` / UTF-8) or ``bytes``.
"""

import ctypes as C
import os

import numpy

from .hpgl_wrap import (_HPGL_B200_IO_TIMING, _HPGL_COKRIGING_M1_PARAMS, _HPGL_COKRIGING_M2_PARAMS, _HPGL_CONT_MASKED_ARRAY, _HPGL_COV_PARAMS, _HPGL_IK_PARAMS, _HPGL_IND_MASKED_ARRAY,
                        _HPGL_MEDIAN_IK_PARAMS, _HPGL_OK_PARAMS, _HPGL_SHAPE, _HPGL_SK_PARAMS, HpglError, _hpgl_so,
                        check_last_error, hpgl_output_handler, hpgl_progress_handler)

__all__ = ["ContProperty", "IndProperty", "SugarboxGrid", "CovarianceModel", "covariance", "ordinary_kriging",
           "simple_kriging", "lvm_kriging", "median_ik", "indicator_kriging", "simple_kriging_weights",
           "simple_cokriging_markI", "simple_cokriging_markII",
           "set_thread_num", "get_thread_num", "set_output_handler", "set_progress_handler", "calc_mean",
           "set_precision", "get_precision", "HpglError", "write_property", "write_gslib_property",
           "load_cont_property", "read_inc_file_float", "read_inc_file_byte", "load_ind_property",
           "get_gslib_property", "io_last_timing"]

_PRECISION = {"fp64": 0, "mixed": 1}


def _c_array(ar_type, size, values):
    if len(values) != size:
        raise RuntimeError("%s values specified for array of %s elements" % (len(values), size))
    return (ar_type * size)(*values)


def _create_hpgl_shape(shape, strides=None):
    if strides is None:
        strides = (1, shape[0], shape[0] * shape[1])
    return _HPGL_SHAPE(data=_c_array(C.c_int, 3, shape), strides=_c_array(C.c_int, 3, strides))


def checkFWA(a):
    """Checks for fortran-order, writable and aligned flags (geo.py:37-41)."""
    assert a.flags["F"] and a.flags["W"] and a.flags["A"]


class ContProperty:
    """Continuous property: float32 values and uint8 informed mask (geo.py:85-107)."""

    def __init__(self, data, mask):
        self.data = numpy.require(data, "float32", "F")
        self.mask = numpy.require(mask, "uint8", "F")

    def validate(self):
        checkFWA(self.data)
        checkFWA(self.mask)
        assert self.data.shape == self.mask.shape

    def fix_shape(self, grid):
        if self.data.ndim != 3 and self.data.size == grid.x * grid.y * grid.z:
            self.data = self.data.reshape((grid.x, grid.y, grid.z), order="F")
        if self.mask.ndim != 3 and self.mask.size == grid.x * grid.y * grid.z:
            self.mask = self.mask.reshape((grid.x, grid.y, grid.z), order="F")

    def __getitem__(self, idx):
        if idx == 0:
            return self.data
        if idx == 1:
            return self.mask
        raise RuntimeError("Index out of range.")


class IndProperty:
    """Indicator property: uint8 category codes, uint8 mask (geo.py:109-130)."""

    def __init__(self, data, mask, indicator_count):
        self.data = numpy.require(data, "uint8", "F")
        self.mask = numpy.require(mask, "uint8", "F")
        self.indicator_count = indicator_count
        if numpy.sum(numpy.bitwise_and(numpy.asarray(mask) > 0, numpy.asarray(data) >= indicator_count)) > 0:
            raise RuntimeError("Property contains some indicators outside of [0..%s] range." % (indicator_count - 1))
        assert numpy.shape(data) == numpy.shape(mask)

    def validate(self):
        checkFWA(self.data)
        checkFWA(self.mask)
        assert self.data.shape == self.mask.shape

    def __getitem__(self, idx):
        if idx == 0:
            return self.data
        if idx == 1:
            return self.mask
        if idx == 2:
            return self.indicator_count
        raise RuntimeError("Index out of range.")


class covariance:
    spherical = 0
    exponential = 1
    gaussian = 2


class SugarboxGrid:
    def __init__(self, x, y, z):
        self.x = x
        self.y = y
        self.z = z


class CovarianceModel:
    """Variogram model (geo.py:157-166): a nugget above the sill is rejected."""

    def __init__(self, type=0, ranges=(0, 0, 0), angles=(0.0, 0.0, 0.0), sill=1.0, nugget=0.0):
        self.type = type
        self.ranges = ranges
        self.angles = angles
        self.sill = sill
        self.nugget = nugget
        if nugget > sill:
            raise Exception("Nugget should be less or equal to Sill")


def _tuple_to_prop(t):
    if isinstance(t, tuple):
        if len(t) == 3:
            return IndProperty(*t)
        if len(t) == 2:
            return ContProperty(*t)
        raise AssertionError("property tuple of length %d" % len(t))
    assert isinstance(t, (ContProperty, IndProperty))
    return t


def _clone_prop(prop):
    """The output starts as a copy of the input (geo.py:232-240); cells the
    algorithm leaves alone keep it."""
    if isinstance(prop, IndProperty):
        return IndProperty(prop.data.copy("F"), prop.mask.copy("F"), prop.indicator_count)
    return ContProperty(prop.data.copy("F"), prop.mask.copy("F"))


def _grid_size(grid):
    return grid.x * grid.y * grid.z


def _cont_array(prop, grid):
    if grid.x * grid.y * grid.z != prop.data.size:
        raise RuntimeError("Invalid data size. Size of data = %s. Size of grid = %s" % (prop.data.size,
                                                                                       _grid_size(grid)))
    return _HPGL_CONT_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_float)),
                                   mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                   shape=_create_hpgl_shape((grid.x, grid.y, grid.z)))


def _ind_array(prop, grid):
    if grid.x * grid.y * grid.z != prop.data.size:
        raise RuntimeError("Invalid data size. Size of data = %s. Size of grid = %s" % (prop.data.size,
                                                                                       _grid_size(grid)))
    return _HPGL_IND_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                  mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                  shape=_create_hpgl_shape((grid.x, grid.y, grid.z)),
                                  indicator_count=prop.indicator_count)


def _kriging_fields(cov_model, radiuses, max_neighbours):
    return dict(covariance_type=cov_model.type, ranges=_c_array(C.c_double, 3, cov_model.ranges),
                angles=_c_array(C.c_double, 3, cov_model.angles), sill=cov_model.sill, nugget=cov_model.nugget,
                radiuses=_c_array(C.c_int, 3, radiuses), max_neighbours=max_neighbours)


class _Precision:
    """Temporarily selects the library precision for one call."""

    def __init__(self, precision):
        self.p = None if precision is None else _PRECISION[precision]

    def __enter__(self):
        if self.p is not None:
            self.old = _hpgl_so.hpgl_b200_get_precision()
            _hpgl_so.hpgl_b200_set_precision(self.p)

    def __exit__(self, *exc):
        if self.p is not None:
            _hpgl_so.hpgl_b200_set_precision(self.old)


def set_precision(precision):
    """Library-wide default: "fp64" (bit-identical to the reference) or "mixed"."""
    _hpgl_so.hpgl_b200_set_precision(_PRECISION[precision])
    check_last_error()


def get_precision():
    return {v: k for k, v in _PRECISION.items()}[_hpgl_so.hpgl_b200_get_precision()]


def ordinary_kriging(prop, grid, radiuses, max_neighbours, cov_model, precision=None):
    prop = _tuple_to_prop(prop)
    out_prop = _clone_prop(prop)
    okp = _HPGL_OK_PARAMS(**_kriging_fields(cov_model, radiuses, max_neighbours))
    inp, outp = _cont_array(prop, grid), _cont_array(out_prop, grid)
    with _Precision(precision):
        _hpgl_so.hpgl_ordinary_kriging(C.byref(inp), C.byref(okp), C.byref(outp))
        check_last_error()
    return out_prop


def simple_kriging(prop, grid, radiuses, max_neighbours, cov_model, mean=None, precision=None):
    prop = _tuple_to_prop(prop)
    out_prop = _clone_prop(prop)
    skp = _HPGL_SK_PARAMS(automatic_mean=(mean is None), mean=(mean if mean is not None else 0),
                          **_kriging_fields(cov_model, radiuses, max_neighbours))
    if grid.x * grid.y * grid.z != prop.data.size:
        raise RuntimeError("Invalid data size. Size of data = %s. Size of grid = %s" % (prop.data.size,
                                                                                       _grid_size(grid)))
    sh = _create_hpgl_shape((grid.x, grid.y, grid.z))
    with _Precision(precision):
        _hpgl_so.hpgl_simple_kriging(prop.data, prop.mask, C.byref(sh), C.byref(skp), out_prop.data, out_prop.mask,
                                     C.byref(sh))
        check_last_error()
    return out_prop


def lvm_kriging(prop, grid, mean_data, radiuses, max_neighbours, cov_model, precision=None):
    prop = _tuple_to_prop(prop)
    out_prop = _clone_prop(prop)
    okp = _HPGL_OK_PARAMS(**_kriging_fields(cov_model, radiuses, max_neighbours))
    mean_data = numpy.require(mean_data, "float32", "F")
    if mean_data.size != prop.data.size or grid.x * grid.y * grid.z != prop.data.size:
        raise RuntimeError("Invalid data size.")
    sh = _create_hpgl_shape((grid.x, grid.y, grid.z))
    with _Precision(precision):
        _hpgl_so.hpgl_lvm_kriging(prop.data, prop.mask, C.byref(sh), mean_data, C.byref(sh), C.byref(okp),
                                  out_prop.data, out_prop.mask, C.byref(sh))
        check_last_error()
    return out_prop


def median_ik(prop, grid, marginal_probs, radiuses, max_neighbours, cov_model, precision=None):
    prop = _tuple_to_prop(prop)
    out_prop = _clone_prop(prop)
    miksp = _HPGL_MEDIAN_IK_PARAMS(marginal_probs=_c_array(C.c_double, 2, marginal_probs),
                                   **_kriging_fields(cov_model, radiuses, max_neighbours))
    inp, outp = _ind_array(prop, grid), _ind_array(out_prop, grid)
    with _Precision(precision):
        _hpgl_so.hpgl_median_ik(C.byref(inp), C.byref(miksp), C.byref(outp))
        check_last_error()
    return out_prop


def _ik_params(data, marginal_probs):
    ikps = []
    for i, ikd in enumerate(data):
        ikps.append(_HPGL_IK_PARAMS(marginal_prob=marginal_probs[i],
                                    **_kriging_fields(ikd["cov_model"], ikd["radiuses"], ikd["max_neighbours"])))
    return _c_array(_HPGL_IK_PARAMS, len(data), ikps)


def indicator_kriging(prop, grid, data, marginal_probs, precision=None):
    """Indicator kriging; with 2 categories it runs median IK with marginal
    probabilities (p0, 1 - p0) and category 0's search, as geo.py:490-501."""
    prop = _tuple_to_prop(prop)
    for i in range(len(data)):
        data[i]["marginal_prob"] = marginal_probs[i]
    if len(data) == 2:
        return median_ik(prop, grid, (data[0]["marginal_prob"], 1 - data[0]["marginal_prob"]), data[0]["radiuses"],
                         data[0]["max_neighbours"], data[0]["cov_model"], precision=precision)
    out_prop = _clone_prop(prop)
    inp, outp = _ind_array(prop, grid), _ind_array(out_prop, grid)
    params = _ik_params(data, marginal_probs)
    with _Precision(precision):
        _hpgl_so.hpgl_indicator_kriging(C.byref(inp), C.byref(outp), params, len(data))
        check_last_error()
    return out_prop


def _cov_fields(cov_model):
    return dict(covariance_type=cov_model.type, ranges=_c_array(C.c_double, 3, cov_model.ranges),
                angles=_c_array(C.c_double, 3, cov_model.angles), sill=cov_model.sill, nugget=cov_model.nugget)


def simple_cokriging_markI(prop, grid, secondary_data, primary_mean, secondary_mean, secondary_variance,
                           correlation_coef, radiuses, max_neighbours, cov_model):
    """Colocated simple cokriging, Markov model I (always the reference's FP64 arithmetic)."""
    prop = _tuple_to_prop(prop)
    secondary_data = _tuple_to_prop(secondary_data)
    out_prop = _clone_prop(prop)
    p = _HPGL_COKRIGING_M1_PARAMS(primary_mean=primary_mean, secondary_mean=secondary_mean,
                                  secondary_variance=secondary_variance, correlation_coef=correlation_coef,
                                  **_kriging_fields(cov_model, radiuses, max_neighbours))
    inp, sec, outp = _cont_array(prop, grid), _cont_array(secondary_data, grid), _cont_array(out_prop, grid)
    _hpgl_so.hpgl_simple_cokriging_mark1(C.byref(inp), C.byref(sec), C.byref(p), C.byref(outp))
    check_last_error()
    return out_prop


def simple_cokriging_markII(grid, primary_data, secondary_data, correlation_coef, radiuses, max_neighbours):
    """Colocated simple cokriging, Markov model II.  ``primary_data`` and
    ``secondary_data`` are dicts with "data" (a property), "mean" and
    "cov_model", as in the reference."""
    prim = _tuple_to_prop(primary_data["data"])
    sec = _tuple_to_prop(secondary_data["data"])
    out_prop = _clone_prop(prim)
    p = _HPGL_COKRIGING_M2_PARAMS(
        primary_cov_params=_HPGL_COV_PARAMS(**_cov_fields(primary_data["cov_model"])),
        secondary_cov_params=_HPGL_COV_PARAMS(**_cov_fields(secondary_data["cov_model"])),
        radiuses=_c_array(C.c_int, 3, radiuses), max_neighbours=max_neighbours,
        primary_mean=primary_data["mean"], secondary_mean=secondary_data["mean"], correlation_coef=correlation_coef)
    inp, secp, outp = _cont_array(prim, grid), _cont_array(sec, grid), _cont_array(out_prop, grid)
    _hpgl_so.hpgl_simple_cokriging_mark2(C.byref(inp), C.byref(secp), C.byref(p), C.byref(outp))
    check_last_error()
    return out_prop


def simple_kriging_weights(center_point, n_x, n_y, n_z, ranges=(100000, 100000, 100000), sill=1,
                           cov_type=covariance.exponential, nugget=None, angles=None):
    """SK weights of one point from explicit neighbour coordinates (geo.py:568-600)."""
    if angles is None:
        angles = (0, 0, 0)
    if nugget is None:
        nugget = 0
    if len(n_x) != len(n_y) or len(n_x) != len(n_z):
        raise RuntimeError("Invalid pointset. %s,%s,%s." % (len(n_x), len(n_y), len(n_z)))
    if nugget > sill:
        raise RuntimeError("Nugget value must be less or equal to Sill value.")
    covp = _HPGL_COV_PARAMS(covariance_type=cov_type, ranges=_c_array(C.c_double, 3, ranges),
                            angles=_c_array(C.c_double, 3, angles), sill=sill, nugget=nugget)
    weights = numpy.zeros(len(n_x), dtype="float32")
    _hpgl_so.hpgl_simple_kriging_weights(_c_array(C.c_float, 3, center_point), numpy.array(n_x, dtype="float32"),
                                         numpy.array(n_y, dtype="float32"), numpy.array(n_z, dtype="float32"),
                                         len(n_x), C.byref(covp), weights)
    check_last_error()
    return weights


def calc_mean(prop):
    """Mean of the informed values (geo.py:370-379)."""
    prop = _tuple_to_prop(prop)
    m = prop.mask.reshape(-1, order="F") == 1
    vals = prop.data.reshape(-1, order="F")[m]
    return float(numpy.sum(vals, dtype=numpy.float64)) / len(vals)


def set_thread_num(num):
    _hpgl_so.hpgl_set_thread_num(num)


def get_thread_num():
    return _hpgl_so.hpgl_get_thread_num()


_handlers = {}


def set_output_handler(handler, param):
    if handler is None:
        _hpgl_so.hpgl_set_output_handler(hpgl_output_handler(), None)
        _handlers.pop("output", None)
    else:
        h = hpgl_output_handler(handler)
        _handlers["output"] = h
        _hpgl_so.hpgl_set_output_handler(h, param)


def set_progress_handler(handler, param):
    if handler is None:
        _hpgl_so.hpgl_set_progress_handler(hpgl_progress_handler(), None)
        _handlers.pop("progress", None)
    else:
        h = hpgl_progress_handler(handler)
        _handlers["progress"] = h
        _hpgl_so.hpgl_set_progress_handler(h, param)


# ---- INC / GSLIB property files ---------------------------------------------

def _fs(name):
    return name if isinstance(name, bytes) else os.fsencode(name)


def _text(name):
    return name if isinstance(name, bytes) else str(name).encode("utf-8")


def _file_shape(data):
    return data.shape if data.ndim == 3 else (data.size, 1, 1)


def _ubyte_ptr(values):
    arr = numpy.ascontiguousarray(numpy.array(values, dtype="uint8").reshape(-1))
    return arr, arr.ctypes.data_as(C.POINTER(C.c_ubyte)), arr.size


def write_property(prop, filename, prop_name, undefined_value, indicator_values=[]):
    """INC file of a property: name line, one value per cell, "/"."""
    prop = _tuple_to_prop(prop)
    sh = _create_hpgl_shape(_file_shape(prop.data))
    if isinstance(prop, ContProperty):
        marr = _HPGL_CONT_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_float)),
                                       mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh)
        _hpgl_so.hpgl_write_inc_file_float(_fs(filename), C.byref(marr), undefined_value, _text(prop_name))
    else:
        marr = _HPGL_IND_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                      mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh,
                                      indicator_count=prop.indicator_count)
        keep, ptr, n = _ubyte_ptr(indicator_values)
        _hpgl_so.hpgl_write_inc_file_byte(_fs(filename), C.byref(marr), int(undefined_value), _text(prop_name), ptr, n)
    check_last_error()


def write_gslib_property(prop, filename, prop_name, undefined_value, indicator_values=[]):
    """GSLIB file of a property: "HPGL saved GSLIB file", "1", name, values."""
    prop = _tuple_to_prop(prop)
    sh = _create_hpgl_shape(_file_shape(prop.data))
    if isinstance(prop, ContProperty):
        marr = _HPGL_CONT_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_float)),
                                       mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh)
        _hpgl_so.hpgl_write_gslib_cont_property(C.byref(marr), _fs(filename), _text(prop_name), undefined_value)
    else:
        marr = _HPGL_IND_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                      mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh,
                                      indicator_count=prop.indicator_count)
        keep, ptr, n = _ubyte_ptr(indicator_values)
        _hpgl_so.hpgl_write_gslib_byte_property(C.byref(marr), _fs(filename), _text(prop_name), undefined_value,
                                                ptr, n)
    check_last_error()


def _count_values(filename):
    n = _hpgl_so.hpgl_b200_inc_count_values(_fs(filename))
    check_last_error()
    return int(n)


def read_inc_file_float(filename, undefined_value, size):
    """`size` = (nx, ny, nz): a ContProperty of that shape (Fortran order)."""
    data = numpy.zeros(size, dtype="float32", order="F")
    mask = numpy.zeros(size, dtype="uint8", order="F")
    _hpgl_so.hpgl_read_inc_file_float(_fs(filename), undefined_value, int(data.size), data, mask)
    check_last_error()
    return ContProperty(data, mask)


def read_inc_file_byte(filename, undefined_value, size, indicator_values):
    """`size` = (nx, ny, nz): an IndProperty whose informed values are the
    indices of the file's values in `indicator_values`."""
    data = numpy.zeros(size, dtype="uint8", order="F")
    mask = numpy.zeros(size, dtype="uint8", order="F")
    values = numpy.array(indicator_values, dtype="uint8").reshape(-1)
    _hpgl_so.hpgl_read_inc_file_byte(_fs(filename), int(undefined_value), int(data.size), data, mask, values,
                                     len(values))
    check_last_error()
    return IndProperty(data, mask, len(indicator_values))


def load_cont_property(filename, undefined_value, size=None):
    if size is None:
        return read_inc_file_float(filename, undefined_value, (_count_values(filename),))
    return read_inc_file_float(filename, undefined_value, size)


def load_ind_property(filename, undefined_value, indicator_values, size=None):
    if size is None:
        return read_inc_file_byte(filename, undefined_value, (_count_values(filename),), indicator_values)
    return read_inc_file_byte(filename, undefined_value, size, indicator_values)


def get_gslib_property(prop_dict, prop_name, undefined_value):
    """(values, informed mask) of one column of a GSLIB table held as a dict."""
    prop = prop_dict[prop_name]
    return (prop, (numpy.asarray(prop) != undefined_value).astype(numpy.uint8))


def io_last_timing():
    """Timings (ms) and sizes of this process's last INC/GSLIB call."""
    t = _HPGL_B200_IO_TIMING()
    _hpgl_so.hpgl_b200_io_last_timing(C.byref(t))
    return {k: getattr(t, k) for k, _ in t._fields_}
