"""A user's whole session through the drop-in entry points, all on the GPU:
an INC file of well data is read (the size counted from the file), its
experimental variogram computed, the cube kriged, and the estimate written
as INC and GSLIB and read back.  The estimate must equal the CPU
restatement's bit for bit (FP64 path), the read-back values the written
floats' "%E" text, and the variogram the restatement's exact sums."""

import numpy as np
import pytest

from hpgl_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_read_variogram_krige_write(tmp_path):
    from hpgl_b200 import cvariogram as CV
    from hpgl_b200.geo_bsd import geo
    job = W.ok_50x50x20(shape=(40, 36, 12), seed=21)
    nx, ny, nz = job["shape"]
    values, mask = job["values"], job["mask"]
    # the well data as an INC file (the reference's writer format)
    src = str(tmp_path / "wells.inc")
    O.write_prop(src, "PORO", values, mask, -99.0)
    prop = geo.load_cont_property(src, -99.0)  # size from the file
    assert prop.data.size == nx * ny * nz
    prop = geo.ContProperty(prop.data.reshape((nx, ny, nz), order="F"), prop.mask.reshape((nx, ny, nz), order="F"))
    read_back, _ = O.read_inc(src, nx * ny * nz, -99.0)
    assert np.array_equal(prop.data.reshape(-1, order="F").view(np.uint32), read_back.view(np.uint32))
    assert np.array_equal(prop.mask.reshape(-1, order="F"), mask)
    # experimental variogram along x
    spec = (2.0, 2.0, 0.8, 8, 0.0, (20.0, 3.0, 2.0), (0.0, 0.0, 0.0))
    t = CV.VariogramSearchTemplate(spec[0], spec[1], spec[2], spec[3], spec[4],
                                   CV.Ellipsoid(*spec[5], *spec[6]))
    sums, counts = CV.CalcVariogramStats(t, hard_data=(prop.data, prop.mask))
    o = O.variograms(O.cv_template(*spec), prop.data, prop.mask)
    assert np.array_equal(counts, o["counts"]) and np.array_equal(sums, o["exact_sums"])
    # ordinary kriging with the reference's own parameters
    p = job["params"][0]
    cm = geo.CovarianceModel(type=p["cov_type"], ranges=p["ranges"], angles=p["angles"], sill=p["sill"],
                             nugget=p["nugget"])
    est = geo.ordinary_kriging(prop, geo.SugarboxGrid(nx, ny, nz), p["radii"], p["max_neighbours"], cm,
                               precision="fp64")
    ojob = dict(job, values=prop.data.reshape(-1, order="F"), mask=prop.mask.reshape(-1, order="F"))
    ref = O.run(ojob, dumps=False)
    assert np.array_equal(est.data.reshape(-1, order="F").view(np.uint32), ref["out"].view(np.uint32))
    assert np.array_equal(est.mask.reshape(-1, order="F"), ref["out_mask"])
    # the estimate written both ways and read back
    out_inc, out_gslib = str(tmp_path / "est.inc"), str(tmp_path / "est.gslib")
    geo.write_property(est, out_inc, "PORO_EST", -99.0)
    geo.write_gslib_property(est, out_gslib, "PORO_EST", -99.0)
    O.write_prop(str(tmp_path / "cpu.inc"), "PORO_EST", est.data.reshape(-1, order="F"),
                 est.mask.reshape(-1, order="F"), -99.0)
    assert open(out_inc, "rb").read() == open(str(tmp_path / "cpu.inc"), "rb").read()
    lines = open(out_gslib).read().splitlines()
    assert lines[:3] == ["HPGL saved GSLIB file", "1", "PORO_EST"] and len(lines) == 3 + nx * ny * nz
    back = geo.read_inc_file_float(out_inc, -99.0, (nx, ny, nz))
    txt = np.array([float(x) for x in open(out_inc).read().split()[1:-1]], np.float32)
    assert np.array_equal(back.data.reshape(-1, order="F").view(np.uint32), txt.view(np.uint32))
