"""ctypes layer of the kriging entry points: the C structs of the library's
ABI (include/hpgl.h, same layouts as the reference's api.h:18-153) and the
argument/return types of each call, following the reference's
geo_bsd/hpgl_wrap.py:18-311.  Loads hpgl_b200/hpgl.so;
there is no fallback when it is missing."""

import ctypes as C
import os

import numpy
import numpy.ctypeslib as NC

hpgl_output_handler = C.CFUNCTYPE(C.c_int, C.c_char_p, C.py_object)
hpgl_progress_handler = C.CFUNCTYPE(C.c_int, C.c_char_p, C.c_int, C.py_object)


class _HPGL_SHAPE(C.Structure):
    _fields_ = [("data", C.c_int * 3), ("strides", C.c_int * 3)]


class _HPGL_CONT_MASKED_ARRAY(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("mask", C.POINTER(C.c_ubyte)), ("shape", _HPGL_SHAPE)]


class _HPGL_IND_MASKED_ARRAY(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_ubyte)), ("mask", C.POINTER(C.c_ubyte)), ("shape", _HPGL_SHAPE),
                ("indicator_count", C.c_int)]


class _HPGL_KRIGING_KIND:
    ordinary = 0
    simple = 1


class _HPGL_UBYTE_ARRAY(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_ubyte)), ("shape", _HPGL_SHAPE)]


class _HPGL_FLOAT_ARRAY(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("shape", _HPGL_SHAPE)]


_KRIGING_FIELDS = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                   ("sill", C.c_double), ("nugget", C.c_double), ("radiuses", C.c_int * 3),
                   ("max_neighbours", C.c_int)]


class _HPGL_OK_PARAMS(C.Structure):
    _fields_ = list(_KRIGING_FIELDS)


class _HPGL_SK_PARAMS(C.Structure):
    _fields_ = _KRIGING_FIELDS + [("automatic_mean", C.c_ubyte), ("mean", C.c_double)]


class _HPGL_MEDIAN_IK_PARAMS(C.Structure):
    _fields_ = _KRIGING_FIELDS + [("marginal_probs", C.c_double * 2)]


class _HPGL_IK_PARAMS(C.Structure):
    _fields_ = _KRIGING_FIELDS + [("marginal_prob", C.c_double)]


class _HPGL_SGS_PARAMS(C.Structure):
    _fields_ = _KRIGING_FIELDS + [("kriging_kind", C.c_int), ("seed", C.c_long), ("min_neighbours", C.c_int)]


class hpgl_non_parametric_cdf_t(C.Structure):
    _fields_ = [("values", C.POINTER(C.c_float)), ("probs", C.POINTER(C.c_float)), ("size", C.c_longlong)]


class _HPGL_COV_PARAMS(C.Structure):
    _fields_ = [("covariance_type", C.c_int), ("ranges", C.c_double * 3), ("angles", C.c_double * 3),
                ("sill", C.c_double), ("nugget", C.c_double)]


class _HPGL_COKRIGING_M1_PARAMS(C.Structure):
    _fields_ = _KRIGING_FIELDS + [("primary_mean", C.c_double), ("secondary_mean", C.c_double),
                                  ("secondary_variance", C.c_double), ("correlation_coef", C.c_double)]


class _HPGL_COKRIGING_M2_PARAMS(C.Structure):
    _fields_ = [("primary_cov_params", _HPGL_COV_PARAMS), ("secondary_cov_params", _HPGL_COV_PARAMS),
                ("radiuses", C.c_int * 3), ("max_neighbours", C.c_int), ("primary_mean", C.c_double),
                ("secondary_mean", C.c_double), ("correlation_coef", C.c_double)]


_LIB_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_hpgl_so = NC.load_library("hpgl", _LIB_DIR)

_F = ["F", "W", "A"]

_hpgl_so.hpgl_get_last_exception_message.restype = C.c_char_p
_hpgl_so.hpgl_get_last_exception_message.argtypes = []
_hpgl_so.hpgl_get_last_error.restype = C.c_int
_hpgl_so.hpgl_get_last_error.argtypes = []

_hpgl_so.hpgl_set_output_handler.restype = None
_hpgl_so.hpgl_set_output_handler.argtypes = [hpgl_output_handler, C.py_object]
_hpgl_so.hpgl_set_progress_handler.restype = None
_hpgl_so.hpgl_set_progress_handler.argtypes = [hpgl_progress_handler, C.py_object]

_hpgl_so.hpgl_ordinary_kriging.restype = None
_hpgl_so.hpgl_ordinary_kriging.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.POINTER(_HPGL_OK_PARAMS),
                                           C.POINTER(_HPGL_CONT_MASKED_ARRAY)]

_hpgl_so.hpgl_simple_kriging.restype = None
_hpgl_so.hpgl_simple_kriging.argtypes = [
    NC.ndpointer(dtype=numpy.float32, flags=_F), NC.ndpointer(dtype=numpy.ubyte, flags=_F),
    C.POINTER(_HPGL_SHAPE), C.POINTER(_HPGL_SK_PARAMS),
    NC.ndpointer(dtype=numpy.float32, flags=_F), NC.ndpointer(dtype=numpy.ubyte, flags=_F),
    C.POINTER(_HPGL_SHAPE)]

_hpgl_so.hpgl_lvm_kriging.restype = None
_hpgl_so.hpgl_lvm_kriging.argtypes = [
    NC.ndpointer(dtype=numpy.float32, flags=_F), NC.ndpointer(dtype=numpy.ubyte, flags=_F),
    C.POINTER(_HPGL_SHAPE), NC.ndpointer(dtype=numpy.float32, flags=_F), C.POINTER(_HPGL_SHAPE),
    C.POINTER(_HPGL_OK_PARAMS), NC.ndpointer(dtype=numpy.float32, flags=_F),
    NC.ndpointer(dtype=numpy.ubyte, flags=_F), C.POINTER(_HPGL_SHAPE)]

_hpgl_so.hpgl_simple_kriging_weights.restype = C.c_int
_hpgl_so.hpgl_simple_kriging_weights.argtypes = [
    (C.c_float * 3), NC.ndpointer(dtype=numpy.float32), NC.ndpointer(dtype=numpy.float32),
    NC.ndpointer(dtype=numpy.float32), C.c_int, C.POINTER(_HPGL_COV_PARAMS), NC.ndpointer(dtype=numpy.float32)]

_hpgl_so.hpgl_median_ik.restype = None
_hpgl_so.hpgl_median_ik.argtypes = [C.POINTER(_HPGL_IND_MASKED_ARRAY), C.POINTER(_HPGL_MEDIAN_IK_PARAMS),
                                    C.POINTER(_HPGL_IND_MASKED_ARRAY)]

_hpgl_so.hpgl_indicator_kriging.restype = None
_hpgl_so.hpgl_indicator_kriging.argtypes = [C.POINTER(_HPGL_IND_MASKED_ARRAY), C.POINTER(_HPGL_IND_MASKED_ARRAY),
                                            C.POINTER(_HPGL_IK_PARAMS), C.c_int]

_hpgl_so.hpgl_simple_cokriging_mark1.restype = None
_hpgl_so.hpgl_simple_cokriging_mark1.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.POINTER(_HPGL_CONT_MASKED_ARRAY),
                                                 C.POINTER(_HPGL_COKRIGING_M1_PARAMS),
                                                 C.POINTER(_HPGL_CONT_MASKED_ARRAY)]
_hpgl_so.hpgl_simple_cokriging_mark2.restype = None
_hpgl_so.hpgl_simple_cokriging_mark2.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.POINTER(_HPGL_CONT_MASKED_ARRAY),
                                                 C.POINTER(_HPGL_COKRIGING_M2_PARAMS),
                                                 C.POINTER(_HPGL_CONT_MASKED_ARRAY)]

_hpgl_so.hpgl_sgs_simulation.restype = None
_hpgl_so.hpgl_sgs_simulation.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.POINTER(_HPGL_SGS_PARAMS),
                                         C.POINTER(hpgl_non_parametric_cdf_t), C.POINTER(C.c_double),
                                         C.POINTER(_HPGL_UBYTE_ARRAY)]
_hpgl_so.hpgl_sgs_lvm_simulation.restype = None
_hpgl_so.hpgl_sgs_lvm_simulation.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.POINTER(_HPGL_SGS_PARAMS),
                                             C.POINTER(hpgl_non_parametric_cdf_t), C.POINTER(_HPGL_FLOAT_ARRAY),
                                             C.POINTER(_HPGL_UBYTE_ARRAY)]
_hpgl_so.hpgl_sis_simulation.restype = None
_hpgl_so.hpgl_sis_simulation.argtypes = [C.POINTER(_HPGL_IND_MASKED_ARRAY), C.POINTER(_HPGL_IK_PARAMS), C.c_int,
                                         C.c_int, C.POINTER(_HPGL_UBYTE_ARRAY)]
_hpgl_so.hpgl_sis_simulation_lvm.restype = None
_hpgl_so.hpgl_sis_simulation_lvm.argtypes = [C.POINTER(_HPGL_IND_MASKED_ARRAY), C.POINTER(_HPGL_IK_PARAMS),
                                             C.POINTER(_HPGL_FLOAT_ARRAY), C.c_int, C.c_int,
                                             C.POINTER(_HPGL_UBYTE_ARRAY), C.c_int]

_hpgl_so.hpgl_read_inc_file_float.restype = None
_hpgl_so.hpgl_read_inc_file_float.argtypes = [C.c_char_p, C.c_float, C.c_int, NC.ndpointer(dtype=numpy.float32, flags=_F),
                                              NC.ndpointer(dtype=numpy.ubyte, flags=_F)]
_hpgl_so.hpgl_read_inc_file_byte.restype = None
_hpgl_so.hpgl_read_inc_file_byte.argtypes = [C.c_char_p, C.c_int, C.c_int, NC.ndpointer(dtype=numpy.ubyte, flags=_F),
                                             NC.ndpointer(dtype=numpy.ubyte, flags=_F),
                                             NC.ndpointer(dtype=numpy.ubyte, flags=_F), C.c_int]
_hpgl_so.hpgl_write_inc_file_float.restype = None
_hpgl_so.hpgl_write_inc_file_float.argtypes = [C.c_char_p, C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.c_float, C.c_char_p]
_hpgl_so.hpgl_write_inc_file_byte.restype = None
_hpgl_so.hpgl_write_inc_file_byte.argtypes = [C.c_char_p, C.POINTER(_HPGL_IND_MASKED_ARRAY), C.c_int, C.c_char_p,
                                              C.POINTER(C.c_ubyte), C.c_int]
_hpgl_so.hpgl_write_gslib_cont_property.restype = None
_hpgl_so.hpgl_write_gslib_cont_property.argtypes = [C.POINTER(_HPGL_CONT_MASKED_ARRAY), C.c_char_p, C.c_char_p,
                                                    C.c_double]
_hpgl_so.hpgl_write_gslib_byte_property.restype = None
_hpgl_so.hpgl_write_gslib_byte_property.argtypes = [C.POINTER(_HPGL_IND_MASKED_ARRAY), C.c_char_p, C.c_char_p,
                                                    C.c_double, C.POINTER(C.c_ubyte), C.c_int]
_hpgl_so.hpgl_b200_inc_count_values.restype = C.c_longlong
_hpgl_so.hpgl_b200_inc_count_values.argtypes = [C.c_char_p]


class _HPGL_B200_IO_TIMING(C.Structure):
    _fields_ = [("ms_file", C.c_double), ("ms_h2d", C.c_double), ("ms_device", C.c_double), ("ms_d2h", C.c_double),
                ("ms_total", C.c_double), ("bytes", C.c_longlong), ("tokens", C.c_longlong)]


_hpgl_so.hpgl_b200_io_last_timing.restype = None
_hpgl_so.hpgl_b200_io_last_timing.argtypes = [C.POINTER(_HPGL_B200_IO_TIMING)]

_hpgl_so.hpgl_set_thread_num.restype = None
_hpgl_so.hpgl_set_thread_num.argtypes = [C.c_int]
_hpgl_so.hpgl_get_thread_num.restype = C.c_int
_hpgl_so.hpgl_get_thread_num.argtypes = []

_hpgl_so.hpgl_b200_set_precision.restype = None
_hpgl_so.hpgl_b200_set_precision.argtypes = [C.c_int]
_hpgl_so.hpgl_b200_get_precision.restype = C.c_int
_hpgl_so.hpgl_b200_get_precision.argtypes = []


class HpglError(RuntimeError):
    """A library call failed; `code` is the HPGL_E_* value."""

    def __init__(self, code, message):
        RuntimeError.__init__(self, message)
        self.code = code


def check_last_error():
    code = _hpgl_so.hpgl_get_last_error()
    if code != 0:
        raise HpglError(code, _hpgl_so.hpgl_get_last_exception_message().decode(errors="replace"))
