"""Host planning of the library (no GPU): the sorted search template must be
the reference's (calc_cov_field, covariance_field.h:62-106) entry for entry,
including the order of equal covariances, which the library reproduces with
a parallel restatement of the reference's sort.  Checked against the oracle
(std::sort itself) on small and large templates."""

import ctypes as C

import numpy as np
import pytest

from hpgl_b200 import native as N
from hpgl_b200 import workloads as W
from oracle import oracle as O


def library_template(p):
    L = N.lib()
    L.hpgl_b200_search_template.restype = C.c_longlong
    L.hpgl_b200_search_template.argtypes = [C.POINTER(N.HpglIkParams), C.POINTER(C.c_int), C.c_longlong]
    prm = N.make_params([p])
    n = L.hpgl_b200_search_template(prm, None, 0)
    assert n >= 0, N.last_error()
    buf = np.zeros(3 * n, dtype=np.int32)
    L.hpgl_b200_search_template(prm, buf.ctypes.data_as(C.POINTER(C.c_int)), n)
    return buf.reshape(n, 3)


CASES = {
    "spherical_iso": W.cov_params(0, (10, 10, 5), radii=(20, 20, 10), max_neighbours=12),
    "exp_az30": W.cov_params(1, (40, 20, 8), angles=(30, 0, 0), sill=1.0, nugget=0.05, radii=(80, 40, 16),
                             max_neighbours=32),
    "gauss_iso_ties": W.cov_params(2, (30, 30, 4), sill=1.0, nugget=0.01, radii=(40, 40, 5), max_neighbours=64),
    "exp_3angles": W.cov_params(1, (25, 15, 10), angles=(20, 10, 5), sill=2.0, nugget=0.3, radii=(40, 30, 20),
                                max_neighbours=16),
    "exp_large_2p5M": W.cov_params(1, (60, 55, 50), sill=1.0, nugget=0.05, radii=(93, 85, 77), max_neighbours=16),
}


@pytest.mark.parametrize("name", list(CASES))
def test_template_equals_reference_order(native_lib, name):
    p = CASES[name]
    ours = library_template(p)
    ref = O.template(p)
    assert ours.shape == ref.shape
    assert np.array_equal(ours, ref)
