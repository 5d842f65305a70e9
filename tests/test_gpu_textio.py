"""INC / GSLIB property files on the GPU against the CPU restatement
(oracle/textio_oracle.cpp), the golden fixtures written by the reference
itself, and the reference's messages: every reader result bit for bit (data,
mask, the error text and the values stored before an error), every written
file byte for byte, through the C ABI and the geo_bsd entry points."""

import ctypes as C
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
import textio_cases as TC

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "textio")


@pytest.fixture(scope="module")
def so():
    from hpgl_b200.geo_bsd import hpgl_wrap
    return hpgl_wrap._hpgl_so


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("inc"))
    return TC.float_cases(d) + TC.byte_cases(d)


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))


def gpu_read(so, path, size, undefined, is_byte=False, values=()):
    """(data, mask, error message or None) through the C ABI."""
    data = np.zeros(size, dtype=np.uint8 if is_byte else np.float32)
    mask = np.zeros(size, dtype=np.uint8)
    if is_byte:
        vals = np.array(values, dtype=np.uint8).reshape(-1)
        so.hpgl_read_inc_file_byte(os.fsencode(path), int(undefined), size, data, mask, vals, len(vals))
    else:
        so.hpgl_read_inc_file_float(os.fsencode(path), undefined, size, data, mask)
    err = None
    if so.hpgl_get_last_error() != 0:
        err = so.hpgl_get_last_exception_message().decode()
    return data, mask, err


def test_reader_matches_oracle_on_every_case(so, cases):
    for c in cases:
        d, m, err = gpu_read(so, c["path"], c["size"], c["undefined"], c["is_byte"], c["values"])
        try:
            od, om = O.read_inc(c["path"], c["size"], c["undefined"], c["is_byte"], c["values"])
            assert err is None, (c["name"], err)
        except O.OracleIoError as e:
            assert err == str(e), (c["name"], err, str(e))
            od, om = e.data, e.mask
        assert _same(d, od), c["name"]
        assert _same(m, om), c["name"]


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_golden(so, path, tmp_path):
    g = np.load(path)
    is_byte = bool(int(g["is_byte"]))
    und = float(g["undefined"])
    if str(g["kind"]) == "read":
        d, m, err = gpu_read(so, path[:-4] + ".inc", int(g["size"]), int(und) if is_byte else und, is_byte,
                             tuple(g["values"]))
        assert err is None
        assert _same(d, g["data"]) and _same(m, g["mask"])
        return
    from hpgl_b200.geo_bsd import geo
    out = str(tmp_path / "w.txt")
    if is_byte:
        prop = geo.IndProperty(g["data"], g["mask"], int(g["indicator_count"]))
        writer = geo.write_property if str(g["fmt"]) == "inc" else geo.write_gslib_property
        writer(prop, out, "FACIES_W", int(und) if str(g["fmt"]) == "inc" else und, list(g["values"]))
    else:
        prop = geo.ContProperty(g["data"], g["mask"])
        writer = geo.write_property if str(g["fmt"]) == "inc" else geo.write_gslib_property
        writer(prop, out, "PORO_W", und)
    with open(out, "rb") as f:
        assert f.read() == g["text"].tobytes()


def test_writers_match_oracle(tmp_path):
    from hpgl_b200.geo_bsd import geo
    rng = np.random.default_rng(3)
    n = 300001
    v = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32).view(np.float32)
    m = (rng.random(n) > 0.25).astype(np.uint8)
    for fmt, writer in (("inc", geo.write_property), ("gslib", geo.write_gslib_property)):
        for und in (-99.0, float("nan"), -0.0):
            a, b = str(tmp_path / "a.txt"), str(tmp_path / "b.txt")
            writer(geo.ContProperty(v, m), a, "PORO", und)
            O.write_prop(b, "PORO", v, m, und, fmt=fmt)
            assert open(a, "rb").read() == open(b, "rb").read(), (fmt, und)
    codes = rng.integers(0, 5, n).astype(np.uint8)
    for fmt, writer in (("inc", geo.write_property), ("gslib", geo.write_gslib_property)):
        for und, values in ((-1, [3, 200, 7, 0, 128]), (17, []), (-99, [9, 8, 7, 6, 5, 4])):
            a, b = str(tmp_path / "a.txt"), str(tmp_path / "b.txt")
            writer(geo.IndProperty(codes, m, 5), a, "FACIES", und, values)
            O.write_prop(b, "FACIES", codes, m, und & 0xff, fmt=fmt, is_byte=True,
                         remap=O.remap_table(values, 5))
            assert open(a, "rb").read() == open(b, "rb").read(), (fmt, und, values)


def test_full_size_write_then_read(so, tmp_path):
    """A 166 x 141 x 225 property (5,266,350 cells): the GPU's file equals
    the restatement's byte for byte, and reading it back equals the
    restatement's reading of it."""
    from hpgl_b200.geo_bsd import geo
    shape = (166, 141, 225)
    n = int(np.prod(shape))
    rng = np.random.default_rng(4)
    v = (rng.lognormal(-1.5, 0.8, n) * np.where(rng.random(n) < 0.5, 1, -1)).astype(np.float32)
    m = (rng.random(n) > 0.8).astype(np.uint8)
    a, b = str(tmp_path / "gpu.inc"), str(tmp_path / "cpu.inc")
    geo.write_property(geo.ContProperty(v.reshape(shape, order="F"), m.reshape(shape, order="F")), a, "PORO", -99.0)
    O.write_prop(b, "PORO", v, m, -99.0)
    assert open(a, "rb").read() == open(b, "rb").read()
    p = geo.read_inc_file_float(a, -99.0, shape)
    od, om = O.read_inc(b, n, -99.0)
    assert _same(p.data.reshape(-1, order="F"), od) and _same(p.mask.reshape(-1, order="F"), om)
    t = geo.io_last_timing()
    assert t["tokens"] == n + 1 and t["ms_device"] > 0  # the values and the closing "/"


def test_many_tiles_comments_long_tokens(so, tmp_path):
    """Several MB of text with comments anywhere, blank lines, tabs, CRLF and
    runs longer than 255 bytes: token boundaries across tiles."""
    rng = np.random.default_rng(5)
    parts = ["-- header comment\n", "PORO\n"]
    for i in range(60000):
        r = rng.random()
        if r < 0.02:
            parts.append("-- comment %d 1 2 3\n" % i)
        elif r < 0.03:
            parts.append("".join(str(int(x)) for x in rng.integers(0, 10, int(rng.integers(200, 900)))) + " ")
        elif r < 0.04:
            parts.append("\r\n\t ")
        else:
            parts.append(" ".join("%.6g" % x for x in rng.normal(0, 3, int(rng.integers(1, 12)))) +
                         (" --x 5 5\n" if rng.random() < 0.05 else "\n"))
    path = str(tmp_path / "big.inc")
    with open(path, "w") as f:
        f.write("".join(parts))
    n = O.inc_count(path)
    assert so.hpgl_b200_inc_count_values(os.fsencode(path)) == n
    d, m, err = gpu_read(so, path, n, -99.0)
    od, om = O.read_inc(path, n, -99.0)
    assert err is None and _same(d, od) and _same(m, om)
    d, m, err = gpu_read(so, path, n + 1000, -99.0)  # past the end: the last value repeats
    od, om = O.read_inc(path, n + 1000, -99.0)
    assert err is None and _same(d, od) and _same(m, om)


def test_geo_bsd_entry_points(tmp_path):
    from hpgl_b200.geo_bsd import geo
    rng = np.random.default_rng(6)
    shape = (7, 5, 3)
    v = rng.normal(size=shape).astype(np.float32)
    msk = (rng.random(shape) > 0.3).astype(np.uint8)
    path = str(tmp_path / "p.inc")
    geo.write_property((np.asfortranarray(v), np.asfortranarray(msk)), path, "PORO", -99.0)
    p = geo.load_cont_property(path, -99.0, shape)
    assert p.data.shape == shape
    assert np.array_equal(p.mask, msk)
    q = geo.load_cont_property(path, -99.0)  # size from the file
    assert q.data.shape == (v.size,)
    assert _same(q.data, p.data.reshape(-1, order="F"))
    codes = rng.integers(0, 3, shape).astype(np.uint8)
    ipath = str(tmp_path / "f.inc")
    geo.write_property(geo.IndProperty(np.asfortranarray(codes), np.asfortranarray(msk), 3), ipath, "F", -1,
                       [10, 20, 30])
    r = geo.load_ind_property(ipath, -1, [10, 20, 30], shape)
    assert np.array_equal(r.mask, msk) and np.array_equal(r.data[msk > 0], codes[msk > 0])
    with pytest.raises(geo.HpglError) as e:
        geo.load_cont_property(str(tmp_path / "missing.inc"), -99.0, shape)
    assert str(e.value) == "read_inc_file_float: Error opening file:%s." % (tmp_path / "missing.inc")
    with pytest.raises(geo.HpglError) as e:
        geo.write_property(p, str(tmp_path / "no" / "dir.inc"), "P", -99.0)
    assert str(e.value) == "open_file_checked: Can't open file '%s'." % (tmp_path / "no" / "dir.inc")



def test_byte_outside_table_is_an_error(so, tmp_path):
    from hpgl_b200.geo_bsd import hpgl_wrap as W
    data = np.array([0, 1, 2, 1], np.uint8)
    mask = np.array([1, 1, 1, 0], np.uint8)
    sh = W._HPGL_SHAPE()
    sh.data[:] = (4, 1, 1)
    arr = W._HPGL_IND_MASKED_ARRAY(data=data.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                   mask=mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh, indicator_count=2)
    path = str(tmp_path / "x.inc")
    so.hpgl_write_inc_file_byte(os.fsencode(path), C.byref(arr), -1, b"F", None, 0)
    assert so.hpgl_get_last_error() != 0
    assert not os.path.exists(path)
