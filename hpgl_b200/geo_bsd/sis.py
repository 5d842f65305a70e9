"""Sequential indicator simulation with the name and arguments of the
reference's geo_bsd/sis.py: ``sis_simulation`` (sis.py:43-77), over
hpgl_sis_simulation / hpgl_sis_simulation_lvm of hpgl_b200/hpgl.so (GPU; no
fallback).

`data` holds one dict per category with "cov_model", "radiuses" and
"max_neighbours"; `marginal_probs` one probability per category, or one
mean cube per category (the LVM form, with the correlogram weights when
use_correlogram is true).  The output starts as a copy of the property, or
an empty property when use_harddata is False.

Differences from the reference, all additive:
* the category dicts are not modified (the reference wrote "marginal_prob"
  into them);
* force_single_thread, force_parallel, use_regions, region_size and
  min_neighbours are accepted and have no effect, as in the reference's
  library;
* every call checks the library's last-error state and raises HpglError.
"""

import ctypes as C

import numpy

from .geo import _clone_prop, _create_hpgl_shape, _ind_array, _tuple_to_prop
from .hpgl_wrap import _HPGL_FLOAT_ARRAY, _HPGL_IK_PARAMS, _HPGL_UBYTE_ARRAY, _hpgl_so, check_last_error

__all__ = ["sis_simulation"]


def _ik_params(data, marginal_probs, is_lvm):
    ps = []
    for i, d in enumerate(data):
        cov = d["cov_model"]
        ps.append(_HPGL_IK_PARAMS(covariance_type=cov.type, ranges=(C.c_double * 3)(*cov.ranges),
                                  angles=(C.c_double * 3)(*cov.angles), sill=cov.sill, nugget=cov.nugget,
                                  radiuses=(C.c_int * 3)(*d["radiuses"]), max_neighbours=d["max_neighbours"],
                                  marginal_prob=0 if is_lvm else marginal_probs[i]))
    return (_HPGL_IK_PARAMS * len(ps))(*ps)


def sis_simulation(prop, grid, data, seed, marginal_probs, use_correlogram=True, mask=None, force_single_thread=False,
                   force_parallel=False, use_harddata=True, use_regions=False, region_size=(), min_neighbours=0):
    """Sequential indicator simulation of an indicator property.

    data: per category {"cov_model", "radiuses", "max_neighbours"}.
    seed: random path and draws.
    marginal_probs: per category a probability, or a mean cube (LVM).
    use_correlogram: the LVM form's correlogram weights.
    mask: None, or an array with 1 in the cells to simulate.
    """
    prop = _tuple_to_prop(prop)
    size = grid.x * grid.y * grid.z
    if len(data) != len(marginal_probs):
        raise ValueError("one marginal probability (or mean cube) per category")
    is_lvm = not numpy.isscalar(marginal_probs[0])
    out_prop = _clone_prop(prop)
    if not use_harddata:
        out_prop.data.fill(0)
        out_prop.mask.fill(0)
    sh = _create_hpgl_shape((grid.x, grid.y, grid.z))
    mask_ptr = None
    if mask is not None:
        mask = numpy.require(mask, "uint8", "F")
        if mask.size != size:
            raise RuntimeError("Invalid mask size.")
        mask_ptr = C.byref(_HPGL_UBYTE_ARRAY(data=mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh))
    ikps = _ik_params(data, marginal_probs, is_lvm)
    arr = _ind_array(out_prop, grid)
    if not is_lvm:
        _hpgl_so.hpgl_sis_simulation(C.byref(arr), ikps, len(data), int(seed), mask_ptr)
    else:
        cubes = [numpy.require(m, "float32", "F") for m in marginal_probs]
        for m in cubes:
            if m.size != size:
                raise RuntimeError("Invalid mean size.")
        means = (_HPGL_FLOAT_ARRAY * len(cubes))(
            *[_HPGL_FLOAT_ARRAY(data=m.ctypes.data_as(C.POINTER(C.c_float)), shape=sh) for m in cubes])
        _hpgl_so.hpgl_sis_simulation_lvm(C.byref(arr), ikps, means, len(data), int(seed), mask_ptr,
                                         int(bool(use_correlogram)))
    check_last_error()
    return out_prop
