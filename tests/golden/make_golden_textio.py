"""Generates the golden fixtures of the INC / GSLIB property files from the
reference's own sources compiled by oracle/build_ref.sh:

* readers: seeded INC files (mixed number formats, comments, CRLF, tabs,
  blank lines, a short file) and what the reference's
  hpgl_read_inc_file_float / hpgl_read_inc_file_byte return for them;
* writers: seeded float and byte properties (with inf, nan, -0, subnormals
  and undefined cells) and the exact files that the reference's
  hpgl_write_inc_file_float/_byte and hpgl_write_gslib_cont/byte_property
  write for them.

    python tests/golden/make_golden_textio.py      # needs the reference build

Writes tests/golden/textio/<case>.inc and <case>.npz."""

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import oracle as O  # noqa: E402
import textio_cases as TC  # noqa: E402

OUT = os.path.join(HERE, "textio")
READ_CASES = ("eclipse_mixed", "crlf_tabs", "short_repeat_last", "prefix_tokens", "long_run_split",
              "comment_in_chunk", "midpoints", "codes", "codes_undef_255")


def float_property(rng, n):
    v = rng.normal(0.0, 1.0, n).astype(np.float32) * np.float32(10.0) ** rng.integers(-40, 39, n).astype(np.float32)
    special = np.array([np.inf, -np.inf, np.nan, -0.0, 0.0, 1e-45, -1e-45, 3.4028235e38, 1234567.5, 1234568.5,
                        0.1, -99.0], np.float32)
    v[: special.size] = special
    mask = (rng.random(n) > 0.2).astype(np.uint8)
    mask[: special.size] = 1
    return v, mask


def main():
    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory() as d:
        for c in TC.float_cases(d) + TC.byte_cases(d):
            if c["name"] not in READ_CASES:
                continue
            assert c["ref_ok"]
            data, mask = O.ref_read_inc(c["path"], c["size"], c["undefined"], c["is_byte"], c["values"])
            with open(c["path"], "rb") as f:
                text = f.read()
            with open(os.path.join(OUT, c["name"] + ".inc"), "wb") as f:
                f.write(text)
            np.savez_compressed(os.path.join(OUT, c["name"] + ".npz"), kind=np.array("read"), size=c["size"],
                                undefined=np.float64(c["undefined"]), is_byte=int(c["is_byte"]),
                                values=np.array(c["values"], np.uint8), data=data, mask=mask)
            print("read", c["name"], c["size"])
        rng = np.random.default_rng(7)
        v, m = float_property(rng, 3000)
        for fmt, und in (("inc", -99.0), ("gslib", -999.25)):
            path = os.path.join(d, "w.txt")
            O.ref_write_prop(path, "PORO_W", v, m, und, fmt=fmt)
            with open(path, "rb") as f:
                text = f.read()
            name = "write_float_" + fmt
            np.savez_compressed(os.path.join(OUT, name + ".npz"), kind=np.array("write"), fmt=np.array(fmt),
                                is_byte=0, undefined=np.float64(und), data=v, mask=m,
                                values=np.zeros(0, np.uint8), indicator_count=0,
                                text=np.frombuffer(text, np.uint8))
            print("write", name, len(text))
        codes = rng.integers(0, 4, 2500).astype(np.uint8)
        cmask = (rng.random(2500) > 0.25).astype(np.uint8)
        for fmt, und, values in (("inc", -1, (10, 20, 200, 7)), ("gslib", -99.0, (1, 2, 3, 4, 5, 6)),
                                 ("inc", 255, ())):
            path = os.path.join(d, "w.txt")
            O.ref_write_prop(path, "FACIES_W", codes, cmask, und, fmt=fmt, is_byte=True, values=values,
                             indicator_count=4)
            with open(path, "rb") as f:
                text = f.read()
            name = "write_byte_%s_%d" % (fmt, len(values))
            np.savez_compressed(os.path.join(OUT, name + ".npz"), kind=np.array("write"), fmt=np.array(fmt),
                                is_byte=1, undefined=np.float64(und), data=codes, mask=cmask,
                                values=np.array(values, np.uint8), indicator_count=4,
                                text=np.frombuffer(text, np.uint8))
            print("write", name, len(text))


if __name__ == "__main__":
    main()
