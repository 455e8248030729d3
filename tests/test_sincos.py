"""Sine and cosine as the GPU path evaluates them for rigid-body rotations
(melody2d_b200/csrc/mel_sincos.h) against an 80-digit decimal evaluation: each must be the double
nearest to the exact value.  The reference turns rigid nodes with glibc's cos and sin
(Code/Body.h:2284-2300), which miss that double for a few arguments in ten thousand (by one unit
in the last place); like x^(-1/2), this is why the oracle's correctly-rounded mode (which uses
mel_sincos.h) is the one the GPU path is compared with bit for bit."""
import ctypes as C
import os
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

from conftest import ROOT

getcontext().prec = 80


def _arctan_inv(x: int) -> Decimal:
    x = Decimal(x)
    s, t, n, sign, x2 = Decimal(0), 1 / x, 1, 1, x * x
    while True:
        term = t / n
        if term < Decimal(10) ** -78:
            return s
        s += sign * term
        t /= x2
        n += 2
        sign = -sign


PI = 16 * _arctan_inv(5) - 4 * _arctan_inv(239)    # Machin's formula


def exact_sincos(x: float):
    d = Decimal(float(x))
    n = (d / (PI / 2)).to_integral_value()
    r = d - n * (PI / 2)
    r2 = r * r
    s, c = Decimal(0), Decimal(0)
    term_s, term_c, k = r, Decimal(1), 0
    while abs(term_s) > Decimal(10) ** -75 or abs(term_c) > Decimal(10) ** -75:
        s += term_s
        c += term_c
        term_s = -term_s * r2 / ((2 * k + 2) * (2 * k + 3))
        term_c = -term_c * r2 / ((2 * k + 1) * (2 * k + 2))
        k += 1
    q = int(n) % 4
    sin_x = [s, c, -s, -c][q]
    cos_x = [c, -s, -c, s][q]
    return float(sin_x), float(cos_x)


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("sincos") / "libsincos.so")
    subprocess.run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                    "-I" + os.path.join(ROOT, "melody2d_b200", "csrc"),
                    os.path.join(ROOT, "tests", "emul", "sincos_shim.c"), "-o", out, "-lm"], check=True)
    L = C.CDLL(out)
    for f in (L.mel_sincos_batch, L.libm_sincos_batch):
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        f.restype = None
    return L


def _run(f, xs):
    s, c = np.empty_like(xs), np.empty_like(xs)
    f(xs.ctypes.data, s.ctypes.data, c.ctypes.data, len(xs))
    return s, c


def test_sincos_correctly_rounded(shim):
    rng = np.random.default_rng(3)
    sgn = rng.choice([-1.0, 1.0], 12000)
    # rigid rotation angles of the workloads are small; cover them densely and add whole turns
    xs = np.concatenate([sgn * 10.0 ** rng.uniform(-12, 0.5, 12000), rng.uniform(-20.0, 20.0, 4000),
                         rng.uniform(-800000.0, 800000.0, 500)])
    ref = np.array([exact_sincos(x) for x in xs])
    s, c = _run(shim.mel_sincos_batch, xs)
    np.testing.assert_array_equal(s, ref[:, 0])
    np.testing.assert_array_equal(c, ref[:, 1])
    gs, gc = _run(shim.libm_sincos_batch, xs)
    for got, want in ((gs, ref[:, 0]), (gc, ref[:, 1])):
        bad = got != want
        # glibc's misses are one unit in the last place, never more
        assert np.all(np.abs(got[bad] - want[bad]) <= np.spacing(np.abs(want[bad])))
    nbad = int((gs != ref[:, 0]).sum() + (gc != ref[:, 1]).sum())
    print("glibc sin/cos misrounded for %d of %d values" % (nbad, 2 * len(xs)))


def test_sincos_special_values(shim):
    xs = np.array([0.0, -0.0, 1e-300, -5e-324, np.pi / 2, np.pi, 1e7, np.inf, np.nan])
    s, c = _run(shim.mel_sincos_batch, xs)
    assert s[0] == 0.0 and not np.signbit(s[0]) and c[0] == 1.0
    assert s[1] == 0.0 and np.signbit(s[1]) and c[1] == 1.0
    assert s[2] == 1e-300 and c[2] == 1.0 and s[3] == -5e-324
    assert (s[4], c[4]) == exact_sincos(np.pi / 2) and (s[5], c[5]) == exact_sincos(np.pi)
    assert s[6] == np.sin(1e7) and c[6] == np.cos(1e7)      # beyond the reduction's range: the C library
    assert np.isnan(s[7]) and np.isnan(c[7]) and np.isnan(s[8]) and np.isnan(c[8])
