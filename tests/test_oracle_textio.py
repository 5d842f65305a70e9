"""The CPU restatement of the INC / GSLIB readers and writers
(oracle/textio_oracle.cpp) against the reference's own entry points compiled
from its sources, and against the committed golden fixtures
(tests/golden/make_golden_textio.py)."""

import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
import textio_cases as TC

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "textio")

# what the reference throws (or, where it never returns, what both readers raise)
EXPECTED_ERRORS = {
    "short_comment_last": "load_floats_into_vector: Unexpected end of data.",
    "slash_early": "load_floats_into_vector: Unexpected end of data.",
    "slash_glued": "load_floats_into_vector: Unexpected end of data.",
    "bad_token": "load_floats_into_vector: Error parsing 'abc' string.",
    "special_tokens": "load_floats_into_vector: Error parsing 'infin' string.",
    "no_name": "read_prop_name: Property name not found.",
    "empty": "read_prop_name: Property name not found.",
    "name_only": "load_floats_into_vector: Unexpected end of data.",
    "codes_bad": "load_floats_into_vector: Error parsing 'x' string.",
    "codes_minus": "load_floats_into_vector: Error parsing '-' string.",
    "high_bytes": "load_floats_into_vector: Error parsing '\u00e9' string.",  # the token's bytes C3 A9
}


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("inc"))
    return TC.float_cases(d) + TC.byte_cases(d)


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))


def test_oracle_reader_errors(cases):
    for c in cases:
        want = EXPECTED_ERRORS.get(c["name"])
        if want is None:
            O.read_inc(c["path"], c["size"], c["undefined"], c["is_byte"], c["values"])
        else:
            with pytest.raises(O.OracleIoError) as e:
                O.read_inc(c["path"], c["size"], c["undefined"], c["is_byte"], c["values"])
            assert str(e.value) == want, c["name"]
            assert not c["ref_ok"]


def test_oracle_partial_values_before_error(cases):
    # the 123 values before the bad token are stored, nothing after it
    c = next(c for c in cases if c["name"] == "bad_token")
    with pytest.raises(O.OracleIoError) as e:
        O.read_inc(c["path"], c["size"], c["undefined"])
    first, _ = O.read_inc(c["path"], 123, c["undefined"])
    assert _same(e.value.data[:123], first)
    assert np.all(e.value.data[123:] == 0) and np.all(e.value.mask == 0)


@pytest.mark.skipif(not O.reference_available(), reason="compiled reference not present")
def test_oracle_reader_matches_compiled_reference(cases):
    n = 0
    for c in cases:
        if not c["ref_ok"]:
            continue
        od, om = O.read_inc(c["path"], c["size"], c["undefined"], c["is_byte"], c["values"])
        rd, rm = O.ref_read_inc(c["path"], c["size"], c["undefined"], c["is_byte"], c["values"])
        assert _same(od, rd) and _same(om, rm), c["name"]
        n += 1
    assert n >= 20


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_oracle_matches_golden(path, tmp_path):
    g = np.load(path)
    if str(g["kind"]) == "read":
        inc = path[:-4] + ".inc"
        und = float(g["undefined"])
        d, m = O.read_inc(inc, int(g["size"]), int(und) if int(g["is_byte"]) else und, bool(int(g["is_byte"])),
                          tuple(g["values"]))
        assert _same(d, g["data"]) and _same(m, g["mask"])
    else:
        out = str(tmp_path / "w.txt")
        is_byte = bool(int(g["is_byte"]))
        und = float(g["undefined"])
        if is_byte:
            table = O.remap_table(list(g["values"]), int(g["indicator_count"]))
            ub = (int(und) & 0xff)
            O.write_prop(out, "FACIES_W", g["data"], g["mask"], ub, fmt=str(g["fmt"]), is_byte=True, remap=table)
        else:
            O.write_prop(out, "PORO_W", g["data"], g["mask"], und, fmt=str(g["fmt"]))
        with open(out, "rb") as f:
            assert f.read() == g["text"].tobytes()


@pytest.mark.skipif(not O.reference_available(), reason="compiled reference not present")
@pytest.mark.parametrize("fmt", ["inc", "gslib"])
def test_oracle_writers_match_compiled_reference(fmt, tmp_path):
    rng = np.random.default_rng(11)
    n = 5000
    bits = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    v = bits.view(np.float32).copy()
    m = (rng.random(n) > 0.3).astype(np.uint8)
    for und in (-99.0, 0.0, 1e30, float("inf")):
        a, b = str(tmp_path / "a.txt"), str(tmp_path / "b.txt")
        O.write_prop(a, "P", v, m, und, fmt=fmt)
        O.ref_write_prop(b, "P", v, m, und, fmt=fmt)
        assert open(a, "rb").read() == open(b, "rb").read()
    codes = rng.integers(0, 3, n).astype(np.uint8)
    for und, values in ((-1, (5, 200, 9)), (-99.0, (1, 2)), (300.0, (7, 8, 9, 10)), (5, ())):
        a, b = str(tmp_path / "a.txt"), str(tmp_path / "b.txt")
        table = O.remap_table(values, 3)
        O.write_prop(a, "F", codes, m, int(und) & 0xff, fmt=fmt, is_byte=True, remap=table)
        O.ref_write_prop(b, "F", codes, m, und, fmt=fmt, is_byte=True, values=values, indicator_count=3)
        assert open(a, "rb").read() == open(b, "rb").read(), (und, values)


def test_oracle_count(cases):
    counts = {c["name"]: O.inc_count(c["path"]) for c in cases if c["name"] not in ("no_name", "empty")}
    assert counts["plain_E"] == 997
    assert counts["slash_early"] == 300
    assert counts["comment_glued"] == 6
    assert counts["name_only"] == 0
    with pytest.raises(O.OracleIoError):
        O.inc_count(next(c for c in cases if c["name"] == "empty")["path"])
