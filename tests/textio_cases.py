"""INC files for the reader tests: each case is a file plus how to read it
(size, undefined value, float or byte, indicator values) and whether the
reference's own reader may be run on it (it must not throw, loop forever or
read an uninitialised buffer there)."""

import os

import numpy as np

_FLOAT_FORMATS = ["%E", "%.4f", "%g", "%.9g", "%.3e", "%d"]


def _fmt(v, fmt):
    if fmt == "%d":
        return "%d" % int(v)
    return fmt % v


def _values(rng, n, undefined, frac_undefined=0.2):
    v = rng.normal(0.25, 0.1, n).astype(np.float32)
    v[rng.random(n) < frac_undefined] = undefined
    return v


def _lines(tokens, per_line, rng, crlf=False, comments=False):
    out = []
    i = 0
    while i < len(tokens):
        k = per_line if per_line else 1 + int(rng.integers(0, 8))
        line = tokens[i:i + k]
        i += k
        sep = "\t" if rng.random() < 0.2 else " " * (1 + int(rng.integers(0, 3)))
        text = sep.join(line)
        if comments and rng.random() < 0.1:
            text += " -- note " + " ".join(tokens[i:i + 2])  # tokens after "--" on this line are skipped
        out.append(text)
        if rng.random() < 0.05:
            out.append("")
    nl = "\r\n" if crlf else "\n"
    return nl.join(out) + nl


def _write(path, text):
    with open(path, "wb") as f:
        f.write(text if isinstance(text, bytes) else text.encode("latin-1"))


def float_cases(d, seed=0):
    rng = np.random.default_rng(seed)
    cases = []

    def add(name, text, size, undefined=-99.0, ref_ok=True, is_byte=False, values=()):
        path = os.path.join(d, name + ".inc")
        _write(path, text)
        cases.append(dict(name=name, path=path, size=size, undefined=undefined, ref_ok=ref_ok, is_byte=is_byte,
                          values=tuple(values)))

    n = 997
    v = _values(rng, n, -99.0)
    toks = ["%E" % x for x in v]
    add("plain_E", "PORO\n" + "\n".join(toks) + "\n/\n", n)
    toks = [_fmt(x, _FLOAT_FORMATS[int(rng.integers(0, 5))]) for x in v]
    add("eclipse_mixed", "-- generated by a test\n-- second comment line\nPORO\n" +
        _lines(toks, 6, rng, comments=True) + "/\n", n)
    add("crlf_tabs", "PERMX\r\n" + _lines(toks, 0, rng, crlf=True) + "/\r\n", n)
    add("extra_after_size", "PORO\n" + " ".join(toks) + " 1 2 3 garbage / more\n", n - 5)
    add("short_repeat_last", "PORO\n" + " ".join(toks[:400]) + "\n", 450)
    add("short_comment_last", "PORO\n" + " ".join(toks[:400]) + "\n-- the end\n", 450, ref_ok=False)
    add("slash_early", "PORO\n" + " ".join(toks[:300]) + "\n/\n" + " ".join(toks[300:]) + "\n", 500, ref_ok=False)
    add("slash_glued", "PORO\n" + " ".join(toks[:300]) + " /x 1 2\n", 302, ref_ok=False)
    add("bad_token", "PORO\n" + " ".join(toks[:123]) + " abc " + " ".join(toks[123:]) + "\n/\n", 600,
        ref_ok=False)
    add("bad_after_size", "PORO\n" + " ".join(toks[:200]) + " abc\n", 200)
    add("prefix_tokens", "PORO\n1.5abc 2e 3e+ .5 5. -0 +7 1,5 3*0.5 0x1p3 0x.8 inf -infinity nan -nan(1) "
        "1e400 1e-400 7.1e-46 00012 1.0E+00x\n/\n", 20)
    add("special_tokens", "PORO\ninfin\n", 1, ref_ok=False)
    long_run = "".join(str(int(d)) for d in rng.integers(0, 10, 600))
    add("long_run_split", "PORO\n1 2 " + long_run + " 4\n", 6)
    comment_chunk = "1" * 255 + "--xyz 9 9\n5"
    add("comment_in_chunk", "PORO\n" + comment_chunk + "\n", 2)
    add("comment_glued", "PORO\n1.0--x 2 -1 3\n--4 5\n6 -- 7\n8\n", 6)
    add("leading_lines", "12 13\n-- c\n   \n  7indented\nNAME rest of line\n1 2 3\n", 3)
    add("leading_lines_ok", "12 13\n-- c\n   \n  7indented\nNAME\n1 2 3\n", 3)
    add("first_byte_newline", "\n\nPORO\n1 2 3\n", 3, ref_ok=False)
    add("long_skipped_line", "1" * 1023 + "\nNOTNAME\nPORO\n4 5\n", 2)
    add("long_name_line", "P" * 1500 + "\n7 8 9\n", 3)
    add("no_name", "1 2 3\n-- x\n", 1, ref_ok=False)
    add("empty", "", 1, ref_ok=False)
    add("name_only", "PORO\n", 3, ref_ok=False)
    add("nul_byte", b"PORO\n1.5\x00abc 2.5\n", 2)
    add("midpoints", "PORO\n" + " ".join([
        "1.00000005960464477539062500000", "1.00000005960464477539062500001",
        "0.000000000000000000000000000000000000000000000700649232162408535461864791644958065640130970938257885878534141944895541342930300743319094181060791015625",
        "340282356779733661637539395458142568448", "340282356779733661637539395458142568447",
        "16777217", "16777219", "9007199254740993", "1.17549435e-38", "0.99999999"]) + "\n", 10)
    add("vt_ff_ws", "PORO\x0b\x0c\n1\x0b2\x0c3\r4\r\n\x0b5\x0c\n", 5)
    add("high_bytes", b"PORO\n1.5\xa0 2\xff\xfe 3 \xc3\xa9 4\n", 4, ref_ok=False)
    add("undefined_nan", "PORO\n1 nan 2 -99 3\n", 5, undefined=float("nan"))
    return cases


def byte_cases(d, seed=1):
    rng = np.random.default_rng(seed)
    cases = []

    def add(name, text, size, undefined=-1, ref_ok=True, values=(0, 1)):
        path = os.path.join(d, name + ".inc")
        _write(path, text)
        cases.append(dict(name=name, path=path, size=size, undefined=undefined, ref_ok=ref_ok, is_byte=True,
                          values=tuple(values)))

    n = 1531
    codes = rng.choice([0, 1, 2, 5, -1], n, p=[0.3, 0.3, 0.1, 0.1, 0.2])
    toks = [str(int(c)) for c in codes]
    add("codes", "FACIES\n" + _lines(toks, 8, rng, comments=True) + "/\n", n, values=(0, 1, 2, 5))
    add("codes_not_in_list", "FACIES\n" + " ".join(toks) + "\n/\n", n, values=(1, 5))
    add("codes_undef_255", "FACIES\n1 255 0 255 300 -1 +4 0x10 12abc 99999999999999999999\n/\n", 10,
        undefined=255, values=(0, 1, 44, 4))
    add("codes_bad", "FACIES\n1 0 x 1\n", 4, ref_ok=False)
    add("codes_short", "FACIES\n1 0 1\n", 7, values=(0, 1))
    add("codes_minus", "FACIES\n- 1\n", 2, ref_ok=False)
    return cases
