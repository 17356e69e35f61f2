"""The story reader's number conversion (starlab_b200/csrc/story_num.h) against
the C library, on the CPU.

The header is host/device code: compiled here by the host compiler into a
small shim, it must give what strtod / strtol give -- bit for bit, with the
same number of characters used -- on every number form the reference's
snapshot reader meets (dyn_io.C:192-200, util_io.C:145-157,
tree_io.C:330): Starlab's own "%.18g" output, other precisions and
exponent forms, exact halfway cases (ties to even), subnormals, overflow,
signs, whitespace, inf/nan, and text that converts nothing.  Forms the
reader reports instead of converting (hexadecimal floats, NaN payloads,
more than 40 significant digits) must be reported, never guessed.
"""
import ctypes
import os
import random
import struct
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(REPO, "starlab_b200", "csrc")

SHIM = r"""
#include "story_num.h"
extern "C" int sn_real(const char *p, long len, double *v, int *err) {
    story::Real r = story::parse_real(p, p + len);
    *v = r.v; *err = r.err; return r.n;
}
extern "C" int sn_long(const char *p, long len, long long *v) {
    story::Long r = story::parse_long(p, p + len);
    *v = r.v; return r.n;
}
"""


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    d = tmp_path_factory.mktemp("story_num")
    src = d / "shim.cpp"
    src.write_text(SHIM)
    lib = d / "libshim.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + HDR, "-o", str(lib), str(src)],
                   check=True)
    L = ctypes.CDLL(str(lib))
    L.sn_real.argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.POINTER(ctypes.c_double),
                          ctypes.POINTER(ctypes.c_int)]
    L.sn_long.argtypes = [ctypes.c_char_p, ctypes.c_long, ctypes.POINTER(ctypes.c_longlong)]
    return L


libc = ctypes.CDLL(None)
libc.strtod.restype = ctypes.c_double
libc.strtod.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
libc.strtol.restype = ctypes.c_long
libc.strtol.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int]


def bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def c_strtod(s):
    b = ctypes.create_string_buffer(s)
    end = ctypes.c_char_p()
    v = libc.strtod(b, ctypes.byref(end))
    return v, ctypes.cast(end, ctypes.c_void_p).value - ctypes.addressof(b)


def ours(shim, s):
    v, e = ctypes.c_double(), ctypes.c_int()
    n = shim.sn_real(s, len(s), ctypes.byref(v), ctypes.byref(e))
    return v.value, n, e.value


def check(shim, strings):
    bad = []
    for s in strings:
        if isinstance(s, str):
            s = s.encode()
        rv, rn = c_strtod(s)
        v, n, err = ours(shim, s)
        assert err == 0, s
        if n != rn or bits(v) != bits(rv):
            bad.append((s, rv, rn, v, n))
    assert not bad, bad[:5]


def rand_doubles(rng, n):
    u = rng.integers(0, 2**63, size=n, dtype=np.uint64) | (rng.integers(0, 2, size=n, dtype=np.uint64) << np.uint64(63))
    x = u.view(np.float64)
    return [float(v) for v in x if np.isfinite(v)]


def test_starlab_output_precisions(shim):
    rng = np.random.default_rng(1)
    xs = rand_doubles(rng, 20000) + list(rng.normal(size=20000) * 10.0 ** rng.integers(-30, 30, size=20000))
    strs = []
    for x in xs:
        for fmt in ("%.18g", "%.17g", "%.16g", "%.15g", "%.6g", "%.25g", "%.21e"):
            strs.append(fmt % x)
    check(shim, strs)


def test_many_digits_and_exponent_forms(shim):
    rng = random.Random(2)
    strs = []
    for _ in range(30000):
        nd = rng.randint(1, 40)
        digits = "".join(rng.choice("0123456789") for _ in range(nd))
        point = rng.randint(0, nd)
        body = digits[:point] + "." + digits[point:] if rng.random() < 0.8 else digits
        e = rng.choice(["", "e%d" % rng.randint(-340, 320), "E+%d" % rng.randint(0, 30), "e-%02d" % rng.randint(0, 99)])
        sign = rng.choice(["", "-", "+"])
        strs.append(sign + body + e)
    check(shim, strs)


def test_halfway_cases_round_to_even(shim):
    getcontext().prec = 200
    rng = np.random.default_rng(3)
    strs = []
    for e in range(20, 90):
        base = 2.0 ** e
        for m in rng.integers(0, 2**52, size=60):
            x = base * (1 + float(m) / 2**52)
            nx = np.nextafter(x, np.inf)
            mid = (Decimal(x) + Decimal(float(nx))) / 2
            t = format(mid.normalize(), "f")
            if len(t.replace(".", "").lstrip("0")) > 40:
                continue
            strs.append(t)
            step = Decimal(10) ** (mid.adjusted() - 38)   # keeps 39-40 significant digits
            strs.append(format(mid + step, "f"))          # just above the midpoint
            strs.append(format(mid - step, "f"))          # just below it
    strs += ["9007199254740993", "9007199254740995", "4503599627370496.5", "4503599627370497.5",
             "1.00000000000000011102230246251565404236316680908203125e0"[:41]]
    check(shim, strs)


def test_up_to_19_digits_near_midpoints(shim):
    """The Eisel-Lemire path (at most 19 significant digits): the closest
    17-, 18- and 19-digit decimals on both sides of the midpoint between a
    double and its upper neighbour, over normal and subnormal doubles and
    every binary exponent, plus exact ties that fit in 19 digits."""
    from decimal import ROUND_CEILING, ROUND_FLOOR
    getcontext().prec = 800
    rng = np.random.default_rng(6)
    xs = [x for x in rand_doubles(rng, 6000) if x > 0]
    xs += list((rng.integers(1, 2**52, size=1000, dtype=np.uint64)).view(np.float64))
    strs = []
    for x in xs:
        nx = float(np.nextafter(x, np.inf))
        if not np.isfinite(nx):
            continue
        mid = (Decimal(float(x)) + Decimal(nx)) / 2
        for nd in (17, 18, 19):
            q = Decimal(1).scaleb(mid.adjusted() - nd + 1)
            for rnd in (ROUND_FLOOR, ROUND_CEILING):
                strs.append("%se%d" % (mid.quantize(q, rounding=rnd).scaleb(-q.adjusted()).to_integral_value(),
                                       q.adjusted()))
    for e in range(53, 63):  # integer ties: 2^e + odd * 2^(e - 53)
        for k in rng.integers(0, 2**51, size=40):
            strs.append(str(2**e + (2 * int(k) + 1) * 2 ** (e - 53)))
    for e in range(48, 53):  # ties with a short binary fraction
        for k in rng.integers(0, 2**51, size=40):
            t = Decimal(2**e) + Decimal(2 * int(k) + 1) * Decimal(2) ** (e - 53)
            strs.append(format(t, "f"))
    check(shim, strs)


def test_subnormals_overflow_and_zero(shim):
    rng = np.random.default_rng(4)
    sub = (rng.integers(1, 2**52, size=3000, dtype=np.uint64)).view(np.float64)
    strs = ["%.17g" % x for x in sub] + ["%.25e" % x for x in sub[:500]]
    strs += ["4.9406564584124654e-324", "2.4703282292062328e-324", "2.4703282292062327e-324",
             "2.4703282292062329e-324", "1e-324", "3e-324", "2.2250738585072011e-308", "2.2250738585072014e-308",
             "1.7976931348623157e308", "1.7976931348623158e308", "1.7976931348623159e308", "1e309", "-1e400",
             "1e-400", "-0", "0e99999999999", "000000000000000000000000000000000000000000001.5", "0.000",
             "1e+", "1e", "5.", ".5", "-.5e1", "  \t\n+3.25x", "1.5e+03abc", "0x", "0xg", "00x1"]
    check(shim, strs)


def test_no_conversion_and_specials(shim):
    check(shim, ["", " ", "-", "+", ".", "abc", "e5", "-e5", ".e1", "in", "na", "infinit",
                 "inf", "-Infinity", "INF rest", "nan", "-NaN", "NAN  "])


def test_reported_forms(shim):
    for s in (b"0x1p3", b"0x.8", b"nan(123)", b"1." + b"1" * 45):
        v, n, err = ours(shim, s)
        assert err == 1, s


def test_strtol(shim):
    cases = ["0", "-17", "  +42x", "9223372036854775807", "9223372036854775808", "-9223372036854775809",
             "123456789012345678901234", "", "-", "x1", " \t7 8"]
    rng = random.Random(5)
    cases += [str(rng.randint(-10**12, 10**12)) for _ in range(2000)]
    for s in cases:
        b = s.encode()
        buf = ctypes.create_string_buffer(b)
        end = ctypes.c_char_p()
        rv = libc.strtol(buf, ctypes.byref(end), 10)
        rn = ctypes.cast(end, ctypes.c_void_p).value - ctypes.addressof(buf)
        v = ctypes.c_longlong()
        n = shim.sn_long(b, len(b), ctypes.byref(v))
        assert (v.value, n) == (rv, rn), s
