"""The correctly rounded sin/cos/asin used by the parity build (and by the
oracle's CR mode) against 120-digit decimal evaluations, on the argument
ranges tracking produces: CSBEND substep angles (|x| < 0.01), slopes for
asin, and RF phases up to 1e6 rad."""
import math
from decimal import Decimal, getcontext

import numpy as np
import pytest

from oracle import pyoracle

getcontext().prec = 130


def _pi():
    def arctan_inv(x):
        x = Decimal(x)
        s, t, n, sign, x2 = Decimal(0), 1 / x, 1, 1, x * x
        while True:
            term = t / n
            if term < Decimal(10) ** -125:
                return s
            s += sign * term
            t /= x2
            n += 2
            sign = -sign
    return 4 * (4 * arctan_inv(5) - arctan_inv(239))


PI = _pi()


def _reduce(x):
    x = Decimal(x)
    k = (x / (2 * PI)).to_integral_value()
    return x - k * 2 * PI


def dsin(x):
    r = _reduce(x)
    t = s = r
    n = 1
    while True:
        t = -t * r * r / ((2 * n) * (2 * n + 1))
        n += 1
        if abs(t) < Decimal(10) ** -120:
            return s
        s += t


def dcos(x):
    r = _reduce(x)
    t = s = Decimal(1)
    n = 1
    while True:
        t = -t * r * r / ((2 * n - 1) * (2 * n))
        n += 1
        if abs(t) < Decimal(10) ** -120:
            return s
        s += t


def dasin(y):
    y = Decimal(y)
    a = Decimal(math.asin(float(y)))
    for _ in range(8):
        a = a - (dsin(a) - y) / dcos(a)
    return a


def dtan(x):
    return dsin(x) / dcos(x)


@pytest.mark.parametrize("kind,lo,hi", [("sin", -0.01, 0.01), ("cos", -0.01, 0.01), ("sin", -1.5, 1.5), ("tan", -0.3, 0.3),
                                        ("cos", -3.0, 3.0), ("sin", -1e6, 1e6), ("asin", -0.01, 0.01),
                                        ("asin", -0.6, 0.6)])
def test_correct_rounding(kind, lo, hi):
    lib = pyoracle.load()
    f = {"sin": lib.orc_cr_sin, "cos": lib.orc_cr_cos, "asin": lib.orc_cr_asin, "tan": lib.orc_cr_tan}[kind]
    ex = {"sin": dsin, "cos": dcos, "asin": dasin, "tan": dtan}[kind]
    rng = np.random.Generator(np.random.Philox(7))
    xs = rng.uniform(lo, hi, 150)
    bad = [x for x in xs if f(float(x)) != float(ex(float(x)))]
    assert not bad, f"{kind}: {len(bad)} of {len(xs)} not correctly rounded, e.g. {bad[:3]}"


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("lo,hi,log_mag", [(2.0 ** -30, 2.0 ** -7, 1), (-2.0 ** -7, 2.0 ** -7, 0),
                                           (2.0 ** -7, 2.0 ** -5, 1), (-0.05, 0.05, 0)])
def test_tiered_paths_agree_with_double_double(kind, lo, hi, log_mag):
    """The tiny- and small-argument paths (plain-double and double-double
    corrections behind a rounding test) against the full double-double
    evaluation on 1e6 arguments per range (kind 3: sin and cos of one
    argument together), and the tiny path's correction within the relative
    error its rounding test assumes (2^-50.7; the test widens by 2^-49)."""
    import ctypes
    lib = pyoracle.load()
    hits, mrel = ctypes.c_long(), ctypes.c_double()
    bad = lib.orc_cr_selftest(kind, lo, hi, log_mag, 1_000_000, 4242 + kind, ctypes.byref(hits), ctypes.byref(mrel))
    assert bad == 0
    assert mrel.value < 2.0 ** -50.7
    if hi <= 2.0 ** -7 and kind < 3 and log_mag == 0:
        assert hits.value > 0.8 * 1_000_000  # the tiny path takes nearly every call


def test_division_with_precomputed_reciprocal_is_ieee():
    """trkcr_div_rcp (Markstein's two FMA corrections from RN(1/b)) against
    the IEEE quotient on 4e6 pairs, a quarter of them on rounding midpoints
    of the quotient and a quarter with divisors of many trailing ones."""
    lib = pyoracle.load()
    assert lib.orc_div_rcp_selftest(4_000_000, 99) == 0


def test_exp_correctly_rounded():
    """trkcr_exp (the Hwang-Lindberg fringe's per-particle exp) against
    120-digit values, on its tiny and general paths."""
    lib = pyoracle.load()
    lib.orc_cr_exp.argtypes = [ctypes_double()]
    lib.orc_cr_exp.restype = ctypes_double()
    rng = np.random.Generator(np.random.Philox(8))
    xs = np.concatenate([rng.uniform(-2.0 ** -7, 2.0 ** -7, 200), rng.uniform(-30, 30, 100)])
    bad = [x for x in xs if lib.orc_cr_exp(float(x)) != float(dexp(float(x)))]
    assert not bad, bad[:3]


@pytest.mark.parametrize("kind", ["sinh", "cosh"])
def test_sinh_cosh_correctly_rounded(kind):
    """trkcr_sinh / trkcr_cosh (the curved-dipole fringe's, EDGE_EFFECTS=5)
    against 120-digit values, on the Taylor path (|x| < 1/8), across the
    switch and on the exponential path up to |x| = 30."""
    lib = pyoracle.load()
    f = getattr(lib, "orc_cr_" + kind)
    f.argtypes = [ctypes_double()]
    f.restype = ctypes_double()
    rng = np.random.Generator(np.random.Philox(9))
    xs = np.concatenate([rng.uniform(-0.125, 0.125, 200), rng.uniform(0.1, 0.2, 60),
                         np.ldexp(rng.uniform(1, 2, 40), rng.integers(-40, -3, 40)), rng.uniform(-30, 30, 100)])
    sign = 1 if kind == "cosh" else -1
    bad = [x for x in xs if f(float(x)) != float((dexp(float(x)) + sign * dexp(-float(x))) / 2)]
    assert not bad, bad[:3]
    assert f(0.0) == (1.0 if kind == "cosh" else 0.0)


def ctypes_double():
    import ctypes
    return ctypes.c_double


def dexp(x):
    x = Decimal(x)
    n = int((x / Decimal(2).ln()).to_integral_value())
    r = x - n * Decimal(2).ln()
    t = s = Decimal(1)
    k = 1
    while True:
        t = t * r / k
        k += 1
        if abs(t) < Decimal(10) ** -125:
            break
        s += t
    return s * (Decimal(2) ** n)
