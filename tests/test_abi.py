"""The C ABI (include/hpgl.h) as a loader sees it, without a GPU:

* every function the header declares is exported by hpgl_b200/hpgl.so;
* the structs have the reference's layouts (sizes and field offsets equal
  to those of the reference's own api.h when its checkout is present, and
  to the ctypes mirrors used by the Python layer);
* argument errors are reported through hpgl_get_last_error /
  hpgl_get_last_exception_message instead of crashing, and a kriging call on
  a machine without a usable GPU fails with HPGL_E_CUDA.
"""

import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from hpgl_b200 import native as N
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hpgl.h")
REF_API = os.path.join(O.reference_src(), "geo_bsd", "hpgl", "api.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(hpgl_[a-z0-9_]+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_t")))


def exported_symbols(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    return set(line.split()[-1] for line in out.splitlines() if " T " in line)


def test_header_symbols_exported(native_lib):
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if n not in exported_symbols(N.LIB_PATH)]
    assert not missing, missing


STRUCTS = ["hpgl_shape_t", "hpgl_cont_masked_array_t", "hpgl_ind_masked_array_t", "hpgl_ok_params_t",
           "hpgl_sk_params_t", "hpgl_cov_params_t", "hpgl_median_ik_params_t", "hpgl_ik_params_t",
           "hpgl_sgs_params_t", "hpgl_cokriging_m1_params_t", "hpgl_cokriging_m2_params_t",
           "hpgl_non_parametric_cdf_t", "hpgl_float_array_t", "hpgl_ubyte_array_t"]
FIELDS = {"hpgl_sk_params_t": ["m_automatic_mean", "m_mean", "m_max_neighbours", "m_radiuses"],
          "hpgl_ik_params_t": ["m_marginal_prob", "m_nugget"],
          "hpgl_median_ik_params_t": ["m_marginal_probs"],
          "hpgl_ind_masked_array_t": ["m_shape", "m_indicator_count"]}


def _layout(header, cxx):
    lines = ['#include <cstdio>', '#include <cstddef>', '#include "%s"' % header, "int main() {"]
    for s in STRUCTS:
        ty = s if cxx else s
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (s, ty))
        for f in FIELDS.get(s, []):
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (s, f, ty, f))
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "l.cpp")
        open(src, "w").write("\n".join(lines))
        exe = os.path.join(d, "l")
        subprocess.run(["g++", "-o", exe, src], check=True, capture_output=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    return dict(line.rsplit(" ", 1) for line in out.splitlines())


def test_struct_layouts_match_reference():
    ours = _layout(HEADER, True)
    from hpgl_b200.geo_bsd import hpgl_wrap as HW
    assert int(ours["hpgl_ok_params_t"]) == C.sizeof(HW._HPGL_OK_PARAMS)
    assert int(ours["hpgl_sk_params_t"]) == C.sizeof(HW._HPGL_SK_PARAMS)
    assert int(ours["hpgl_ik_params_t"]) == C.sizeof(HW._HPGL_IK_PARAMS)
    assert int(ours["hpgl_median_ik_params_t"]) == C.sizeof(HW._HPGL_MEDIAN_IK_PARAMS)
    assert int(ours["hpgl_ind_masked_array_t"]) == C.sizeof(HW._HPGL_IND_MASKED_ARRAY)
    if os.path.exists(REF_API):
        ref = _layout(REF_API, True)
        assert ours == ref


def _job(**kw):
    from hpgl_b200 import workloads as W
    j = W.ok_50x50x20(shape=(8, 8, 4))
    j.update(kw)
    return j


def test_invalid_params_reported(native_lib):
    j = _job()
    j["params"] = [dict(j["params"][0], ranges=(0.0, 10.0, 5.0))]
    with pytest.raises(N.HpglError) as e:
        N.krige(j)
    assert e.value.code == N.HPGL_E_INVALID
    assert "non-zero" in str(e.value)
    j["params"] = [dict(j["params"][0], ranges=(10.0, 10.0, 5.0), max_neighbours=65)]
    with pytest.raises(N.HpglError) as e:
        N.krige(j)
    assert e.value.code == N.HPGL_E_UNSUPPORTED


def test_reference_entry_point_sets_last_error(native_lib):
    from hpgl_b200.geo_bsd import geo
    prop = geo.ContProperty(np.zeros(64, np.float32), np.zeros(64, np.uint8))
    cm = geo.CovarianceModel(type=0, ranges=(0, 1, 1))
    with pytest.raises(geo.HpglError) as e:
        geo.ordinary_kriging(prop, geo.SugarboxGrid(4, 4, 4), (2, 2, 2), 4, cm)
    assert e.value.code == N.HPGL_E_INVALID


def test_no_gpu_is_an_error_not_a_fallback(native_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(N.HpglError) as e:
        N.krige(_job())
    assert e.value.code == N.HPGL_E_CUDA


def test_simulation_entry_points_reject_null_arguments(native_lib):
    L = native_lib
    L.hpgl_sis_simulation(None, None, 0, 0, None)
    assert L.hpgl_get_last_error() == N.HPGL_E_INVALID
    L.hpgl_sis_simulation_lvm(None, None, None, 2, 0, None, 1)
    assert L.hpgl_get_last_error() == N.HPGL_E_INVALID
    L.hpgl_sgs_simulation(None, None, None, None, None)
    assert L.hpgl_get_last_error() == N.HPGL_E_INVALID


# ---- the experimental-variogram ABI (include/cvariogram.h) -------------------------

CV_HEADER = os.path.join(ROOT, "include", "cvariogram.h")
REF_CV_API = os.path.join(O.reference_src(), "geo_bsd", "_cvariogram", "api.h")
CV_STRUCTS = ["vector_t", "ellipsoid_t", "variogram_search_template_t", "cont_point_set_t", "hard_data_t",
              "float_data_t"]


def test_cvariogram_symbols_exported(native_lib):
    text = re.sub(r"/\*.*?\*/", "", open(CV_HEADER).read(), flags=re.S)
    names = sorted(set(re.findall(r"\b([a-z_0-9]+)\s*\(", text)) - {"defined"})
    for want in ("fill_ellipsoid_directions", "calc_variograms", "calc_variograms_from_point_set",
                 "cvar_stack_layers", "hpgl_b200_variogram_stats"):
        assert want in names
    missing = [n for n in names if n not in exported_symbols(N.LIB_PATH)]
    assert not missing, missing


def _cv_layout(header):
    lines = ['#include <cstdio>', '#include "%s"' % header, "int main() {"]
    for s in CV_STRUCTS:
        lines.append('printf("%s %%zu\\n", sizeof(struct %s));' % (s, s))
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "l.cpp")
        open(src, "w").write("\n".join(lines))
        exe = os.path.join(d, "l")
        subprocess.run(["g++", "-o", exe, src], check=True, capture_output=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    return dict(line.rsplit(" ", 1) for line in out.splitlines())


def test_cvariogram_struct_layouts():
    ours = _cv_layout(CV_HEADER)
    from hpgl_b200 import cvariogram as CVP
    assert int(ours["variogram_search_template_t"]) == C.sizeof(CVP.variogram_search_template_t)
    assert int(ours["hard_data_t"]) == C.sizeof(CVP.hard_data_t)
    assert int(ours["cont_point_set_t"]) == C.sizeof(CVP.cont_point_set_t)
    assert int(ours["float_data_t"]) == C.sizeof(CVP.float_data_t)
    if os.path.exists(REF_CV_API):
        assert ours == _cv_layout(REF_CV_API)


def test_ellipsoid_directions_on_the_host(native_lib):
    from hpgl_b200 import cvariogram as CVP
    from oracle import oracle as O
    for angles in ((40.0, 50.0, 60.0), (320.0, 0.0, 0.0), (0.0, 90.0, 0.0)):
        e = CVP.Ellipsoid(10, 20, 30, *angles).ell
        t = O.cv_template(1, 1, 1, 1, 0, (10, 20, 30), angles)
        for k in ("direction1", "direction2", "direction3"):
            assert list(getattr(e, k).data) == list(getattr(t.ellipsoid, k).data)


def test_file_and_variogram_calls_need_the_gpu(native_lib, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from hpgl_b200 import cvariogram as CVP
    from hpgl_b200.geo_bsd import geo
    path = str(tmp_path / "p.inc")
    with open(path, "w") as f:
        f.write("PORO\n1 2 3\n/\n")
    with pytest.raises(geo.HpglError) as e:
        geo.load_cont_property(path, -99.0, (3, 1, 1))
    assert e.value.code == N.HPGL_E_CUDA
    t = CVP.VariogramSearchTemplate(1, 1, 0.5, 4, 0, CVP.Ellipsoid(10, 2, 2, 0, 0, 0))
    v = np.ones((4, 4, 2), np.float32)
    with pytest.raises(geo.HpglError) as e:
        CVP.CalcVariograms(t, (v, np.ones(v.shape, np.uint8)))
    assert e.value.code == N.HPGL_E_CUDA
