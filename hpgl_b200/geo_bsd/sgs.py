"""Sequential Gaussian simulation with the name and arguments of the
reference's geo_bsd/sgs.py: ``sgs_simulation`` (sgs.py:43-118) and
``normed_cov_model`` (:34-41), over hpgl_sgs_simulation /
hpgl_sgs_lvm_simulation of hpgl_b200/hpgl.so (GPU; no fallback).

The covariance model is normalised to a unit sill-minus-nugget, the output
starts as a copy of the property (or an empty property when use_harddata is
False), and a varying `mean` array selects the LVM form.  Simple kriging runs
with mean 0 whatever `mean` is, as in the reference's library.

Differences from the reference, all additive:
* ``cdf_data`` may be None (no transform; the reference's wrapper built the
  CDF structure unconditionally and failed on None), a CdfData, or a property
  (or (data, mask) tuple) whose CDF ``calc_cdf`` computes;
* use_regions, region_size, force_single_thread, force_parallel and
  min_neighbours are accepted and have no effect, as in the reference's
  library;
* every call checks the library's last-error state and raises HpglError.
"""

import ctypes as C

import numpy

from .cdf import CdfData, calc_cdf
from .geo import CovarianceModel, _clone_prop, _cont_array, _create_hpgl_shape, _tuple_to_prop
from .hpgl_wrap import (_HPGL_FLOAT_ARRAY, _HPGL_KRIGING_KIND, _HPGL_SGS_PARAMS, _HPGL_UBYTE_ARRAY, _hpgl_so,
                        check_last_error, hpgl_non_parametric_cdf_t)

__all__ = ["sgs_simulation", "normed_cov_model"]


def normed_cov_model(cov_model):
    coef = cov_model.sill - cov_model.nugget
    return CovarianceModel(cov_model.type, cov_model.ranges, cov_model.angles, cov_model.sill / coef,
                           cov_model.nugget / coef)


def _empty_clone(prop):
    """geo.py:220-230: same shapes, every cell zero and uninformed."""
    out = _clone_prop(prop)
    out.data.fill(0)
    out.mask.fill(0)
    return out


def _shape(grid):
    return _create_hpgl_shape((grid.x, grid.y, grid.z))


def _cdf(cdf_data):
    if cdf_data is None:
        return None
    if not isinstance(cdf_data, CdfData):
        cdf_data = calc_cdf(_tuple_to_prop(cdf_data))
    values = numpy.ascontiguousarray(cdf_data.values, dtype=numpy.float32)
    probs = numpy.ascontiguousarray(cdf_data.probs, dtype=numpy.float32)
    if values.size != probs.size:
        raise ValueError("CDF values and probabilities differ in length")
    c = hpgl_non_parametric_cdf_t(values=values.ctypes.data_as(C.POINTER(C.c_float)),
                                  probs=probs.ctypes.data_as(C.POINTER(C.c_float)), size=values.size)
    return c, (values, probs)


def sgs_simulation(prop, grid, cdf_data, radiuses, max_neighbours, cov_model, seed, kriging_type="sk", mean=None,
                   use_harddata=True, use_regions=False, region_size=None, mask=None, force_single_thread=False,
                   force_parallel=False, min_neighbours=0, **params):
    """Sequential Gaussian simulation of a continuous property.

    cdf_data: None, CdfData, or a property whose CDF is used for the
        normal-score transform.
    radiuses, max_neighbours, cov_model: search and variogram.
    seed: random path and draws.
    kriging_type: "sk" (mean 0) or "ok".
    mean: None or a scalar (stationary), or an array (locally varying mean).
    use_harddata: False simulates from an empty property.
    mask: None, or an array with 1 in the cells to simulate.
    """
    prop = _tuple_to_prop(prop)
    size = grid.x * grid.y * grid.z
    if prop.data.size != size:
        raise RuntimeError("Invalid data size. Size of data = %s. Size of grid = %s" % (prop.data.size, size))
    cov_model = normed_cov_model(cov_model)
    out_prop = _clone_prop(prop) if use_harddata else _empty_clone(prop)
    sgsp = _HPGL_SGS_PARAMS(covariance_type=cov_model.type, ranges=(C.c_double * 3)(*cov_model.ranges),
                            angles=(C.c_double * 3)(*cov_model.angles), sill=cov_model.sill,
                            nugget=cov_model.nugget, radiuses=(C.c_int * 3)(*radiuses),
                            max_neighbours=max_neighbours,
                            kriging_kind={"sk": _HPGL_KRIGING_KIND.simple, "ok": _HPGL_KRIGING_KIND.ordinary}[
                                kriging_type],
                            seed=seed, min_neighbours=min_neighbours)
    cdf = _cdf(cdf_data)
    cdf_ptr = C.byref(cdf[0]) if cdf is not None else None
    mask_ptr = None
    if mask is not None:
        mask = numpy.require(mask, "uint8", "F")
        if mask.size != size:
            raise RuntimeError("Invalid mask size.")
        mask_ptr = C.byref(_HPGL_UBYTE_ARRAY(data=mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=_shape(grid)))
    arr = _cont_array(out_prop, grid)
    if mean is None or numpy.isscalar(mean):
        mean_ptr = C.byref(C.c_double(mean)) if mean is not None else None
        _hpgl_so.hpgl_sgs_simulation(C.byref(arr), C.byref(sgsp), cdf_ptr, mean_ptr, mask_ptr)
    else:
        mean = numpy.require(mean, "float32", "F")
        if mean.size != size:
            raise RuntimeError("Invalid mean size.")
        fa = _HPGL_FLOAT_ARRAY(data=mean.ctypes.data_as(C.POINTER(C.c_float)), shape=_shape(grid))
        _hpgl_so.hpgl_sgs_lvm_simulation(C.byref(arr), C.byref(sgsp), cdf_ptr, C.byref(fa), mask_ptr)
    check_last_error()
    return out_prop
