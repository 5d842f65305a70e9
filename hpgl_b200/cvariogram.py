"""Experimental variograms with the names and arguments of the reference's
geo_bsd/cvariogram.py (Python 2): ``Ellipsoid`` (cvariogram.py:99-111),
``VariogramSearchTemplate`` (:114-126), ``CalcVariograms`` (:129-153),
``CalcVariogramsFromPointSet`` (:155-177), ``CStackLayers`` (:186-200), over
the C ABI of include/cvariogram.h exported by hpgl_b200/hpgl.so (the
reference loads a separate _cvariogram library).  The variograms run on the
GPU; there is no fallback when the library is missing.

Differences from the reference:
* ``CalcVariogramsFromPointSet`` reads the point set as a dict of "X", "Y",
  "Z" and "Property" arrays (the reference's version calls the dict and uses
  an undefined name, so it never ran);
* every call checks the library's last-error state and raises HpglError;
* ``CalcVariogramStats`` returns the per-lag pair counts and sums as well.
"""

import ctypes as C

import numpy
import numpy.ctypeslib as NC

from .geo_bsd.hpgl_wrap import _hpgl_so as cvar
from .geo_bsd.hpgl_wrap import HpglError, check_last_error

__all__ = ["Ellipsoid", "VariogramSearchTemplate", "CalcVariograms", "CalcVariogramsFromPointSet",
           "CalcVariogramStats", "CStackLayers", "HpglError"]


class vector_t(C.Structure):
    _fields_ = [("data", C.c_double * 3)]


class ellipsoid_t(C.Structure):
    _fields_ = [("direction1", vector_t), ("direction2", vector_t), ("direction3", vector_t), ("R1", C.c_double),
                ("R2", C.c_double), ("R3", C.c_double)]


class variogram_search_template_t(C.Structure):
    _fields_ = [("lag_width", C.c_double), ("lag_separation", C.c_double), ("tol_distance", C.c_double),
                ("num_lags", C.c_int), ("first_lag_distance", C.c_double), ("ellipsoid", ellipsoid_t)]


class hard_data_t(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("mask", C.POINTER(C.c_ubyte)), ("data_shape", C.c_int * 3),
                ("data_strides", C.c_int * 3), ("mask_shape", C.c_int * 3), ("mask_strides", C.c_int * 3)]


class cont_point_set_t(C.Structure):
    _fields_ = [("xs", C.POINTER(C.c_float)), ("ys", C.POINTER(C.c_float)), ("zs", C.POINTER(C.c_float)),
                ("values", C.POINTER(C.c_float)), ("values_count", C.c_int)]


class float_data_t(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("data_shape", C.c_int * 3), ("data_strides", C.c_int * 3)]


cvar.fill_ellipsoid_directions.restype = None
cvar.fill_ellipsoid_directions.argtypes = [C.POINTER(ellipsoid_t), C.c_double, C.c_double, C.c_double]
cvar.calc_variograms.restype = None
cvar.calc_variograms.argtypes = [C.POINTER(variogram_search_template_t), C.POINTER(hard_data_t),
                                 NC.ndpointer(dtype=numpy.float32), C.c_int, C.c_int]
cvar.calc_variograms_from_point_set.restype = None
cvar.calc_variograms_from_point_set.argtypes = [C.POINTER(variogram_search_template_t), C.POINTER(cont_point_set_t),
                                                NC.ndpointer(dtype=numpy.float32), C.c_int]
cvar.cvar_stack_layers.restype = None
cvar.cvar_stack_layers.argtypes = [C.POINTER(float_data_t), C.POINTER(C.c_int), C.c_int, C.c_int, C.c_float, C.c_int,
                                   C.POINTER(float_data_t)]
cvar.hpgl_b200_variogram_stats.restype = C.c_int
cvar.hpgl_b200_variogram_stats.argtypes = [C.POINTER(variogram_search_template_t), C.POINTER(hard_data_t),
                                           C.POINTER(cont_point_set_t), C.c_int, C.c_int,
                                           NC.ndpointer(dtype=numpy.float64), NC.ndpointer(dtype=numpy.int64)]


def _strides(array):
    return tuple(s // array.itemsize for s in array.strides)


def _c_array(t, size, values):
    return (t * size)(*values)


class Ellipsoid:
    """Radii and rotations (degrees) of the search tunnel (cvariogram.py:99-111)."""

    def __init__(self, R1, R2, R3, azimuth, dip, rotation):
        self.ell = ellipsoid_t(R1=R1, R2=R2, R3=R3)
        cvar.fill_ellipsoid_directions(C.byref(self.ell), azimuth, dip, rotation)
        check_last_error()


class VariogramSearchTemplate:
    """Lag layout and tunnel (cvariogram.py:114-126)."""

    def __init__(self, lag_width, lag_separation, tol_distance, num_lags, first_lag_distance, ellipsoid):
        self.templ = variogram_search_template_t(lag_width=lag_width, lag_separation=lag_separation,
                                                 tol_distance=tol_distance, num_lags=num_lags,
                                                 first_lag_distance=first_lag_distance, ellipsoid=ellipsoid.ell)
        self.num_lags = num_lags
        self.lag_separation = lag_separation


def _hard_data(hard_data):
    data = numpy.asarray(hard_data[0], dtype=numpy.float32)
    mask = numpy.asarray(hard_data[1], dtype=numpy.uint8)
    if data.ndim != 3 or mask.ndim != 3:
        raise ValueError("hard data must be 3-D arrays")
    hd = hard_data_t(data=data.ctypes.data_as(C.POINTER(C.c_float)), mask=mask.ctypes.data_as(C.POINTER(C.c_ubyte)),
                     data_shape=_c_array(C.c_int, 3, data.shape), mask_shape=_c_array(C.c_int, 3, mask.shape),
                     data_strides=_c_array(C.c_int, 3, _strides(data)),
                     mask_strides=_c_array(C.c_int, 3, _strides(mask)))
    return hd, (data, mask)


def _point_set(point_set):
    arrs = [numpy.ascontiguousarray(point_set[k], dtype=numpy.float32) for k in ("X", "Y", "Z", "Property")]
    ps = cont_point_set_t(xs=arrs[0].ctypes.data_as(C.POINTER(C.c_float)),
                          ys=arrs[1].ctypes.data_as(C.POINTER(C.c_float)),
                          zs=arrs[2].ctypes.data_as(C.POINTER(C.c_float)),
                          values=arrs[3].ctypes.data_as(C.POINTER(C.c_float)), values_count=arrs[3].size)
    return ps, arrs


def _borders(templ):
    return numpy.arange(templ.num_lags) * float(templ.lag_separation)


def CalcVariograms(templ, hard_data, percent=100):
    """(lag borders, semivariances) of (values, mask) 3-D arrays."""
    variogram = numpy.zeros(templ.num_lags, dtype="float32")
    hd, keep = _hard_data(hard_data)
    cvar.calc_variograms(C.byref(templ.templ), C.byref(hd), variogram, variogram.size, int(percent))
    check_last_error()
    return (_borders(templ), variogram)


def CalcVariogramsFromPointSet(templ, point_set, variogram=None):
    """(lag borders, semivariances) of a point set {"X", "Y", "Z", "Property"}."""
    variogram = numpy.zeros(templ.num_lags, dtype="float32")
    ps, keep = _point_set(point_set)
    cvar.calc_variograms_from_point_set(C.byref(templ.templ), C.byref(ps), variogram, variogram.size)
    check_last_error()
    return (_borders(templ), variogram)


def CalcVariogramStats(templ, hard_data=None, point_set=None, percent=100):
    """Per-lag (sums of squared differences, pair counts) of either form."""
    sums = numpy.zeros(templ.num_lags, dtype=numpy.float64)
    counts = numpy.zeros(templ.num_lags, dtype=numpy.int64)
    keep = None
    if point_set is not None:
        ps, keep = _point_set(point_set)
        rc = cvar.hpgl_b200_variogram_stats(C.byref(templ.templ), None, C.byref(ps), templ.num_lags, int(percent),
                                            sums, counts)
    else:
        hd, keep = _hard_data(hard_data)
        rc = cvar.hpgl_b200_variogram_stats(C.byref(templ.templ), C.byref(hd), None, templ.num_lags, int(percent),
                                            sums, counts)
    if rc != 0:
        check_last_error()
    return sums, counts


def _float_data(array):
    a = numpy.asarray(array)
    shape = list(a.shape) + [1] * (3 - a.ndim)
    strides = list(_strides(a)) + [0] * (3 - a.ndim)
    return float_data_t(data=a.ctypes.data_as(C.POINTER(C.c_float)), data_shape=_c_array(C.c_int, 3, shape),
                        data_strides=_c_array(C.c_int, 3, strides))


def CStackLayers(layers, markers, nz, scalez, blank_value, result):
    """Fills `result` (3-D float32) with layer markers from thickness maps."""
    for a in list(layers) + [result]:
        if numpy.asarray(a).dtype != numpy.float32:
            raise ValueError("layers and result must be float32")
    layers2 = [_float_data(l) for l in layers]
    cvar.cvar_stack_layers(_c_array(float_data_t, len(layers2), layers2), _c_array(C.c_int, len(markers), markers),
                           len(layers2), nz, scalez, blank_value, C.byref(_float_data(result)))
    check_last_error()
    return result
