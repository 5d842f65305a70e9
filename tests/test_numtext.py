"""The number <-> text conversions that the INC / GSLIB kernels run
(hpgl_b200/csrc/numtext.cuh), built for the host, against the C library
calls the reference makes: sscanf("%f"), sscanf("%d"), snprintf("%E"),
snprintf("%d").  Tokens come from seeded generators of random characters,
decimal strings, printed floats, decimal expansions of the halfway points
between floats (short and up to 200 digits, exact and nudged), hex floats
and 100-255 digit strings."""

import ctypes as C
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def nt(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("nt") / "numtext_check.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", out,
                    os.path.join(HERE, "numtext_check.cpp")], check=True, capture_output=True)
    lib = C.CDLL(out)
    lib.nt_fuzz_f32.restype = C.c_long
    lib.nt_fuzz_f32.argtypes = [C.c_ulonglong, C.c_long, C.c_int, C.c_char_p, C.c_int]
    lib.nt_fuzz_int.restype = C.c_long
    lib.nt_fuzz_int.argtypes = [C.c_ulonglong, C.c_long, C.c_char_p, C.c_int]
    lib.nt_check_format.restype = C.c_long
    lib.nt_check_format.argtypes = [C.c_ulonglong, C.c_ulonglong, C.c_ulonglong, C.c_long, C.c_char_p, C.c_int]
    lib.nt_check_format_d.restype = C.c_long
    lib.nt_check_format_d.argtypes = [C.c_char_p, C.c_int]
    return lib


@pytest.mark.parametrize("mode", range(7))
def test_scan_f32_matches_sscanf(nt, mode):
    buf = C.create_string_buffer(8192)
    bad = nt.nt_fuzz_f32(1234 + mode, 150000, mode, buf, 8192)
    assert bad == 0, buf.value.decode(errors="replace")


def test_scan_int_matches_sscanf(nt):
    buf = C.create_string_buffer(8192)
    bad = nt.nt_fuzz_int(99, 300000, buf, 8192)
    assert bad == 0, buf.value.decode(errors="replace")


def test_format_E_matches_snprintf(nt):
    buf = C.create_string_buffer(8192)
    bad = nt.nt_check_format(5, 0, 0, 1000000, buf, 8192)  # random bit patterns, 1/8 subnormal
    assert bad == 0, buf.value.decode(errors="replace")
    # every 4099th pattern over the whole range, and the low subnormals and
    # the binades next to the powers of ten exhaustively
    bad = nt.nt_check_format(0, 1 << 32, 4099, 0, buf, 8192)
    assert bad == 0, buf.value.decode(errors="replace")
    bad = nt.nt_check_format(0, 200000, 1, 0, buf, 8192)
    assert bad == 0, buf.value.decode(errors="replace")
    for b in (0x3f800000, 0x41200000, 0x42c80000, 0x49742400, 0x4b189680):  # 1, 10, 100, 1e6, 1e7
        bad = nt.nt_check_format(b - 50000, b + 50000, 1, 0, buf, 8192)
        assert bad == 0, buf.value.decode(errors="replace")


def test_format_d_matches_snprintf(nt):
    buf = C.create_string_buffer(1024)
    assert nt.nt_check_format_d(buf, 1024) == 0, buf.value.decode()
