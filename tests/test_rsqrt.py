"""x^(-1/2) as the GPU path evaluates it (melody2d_b200/csrc/mel_rsqrt.h) against a 60-digit
decimal evaluation: it must be the double nearest to 1/sqrt(x) for every sample.  glibc's
pow(x, -0.5), which the reference calls, misses that double for a small fraction of arguments
(always by one unit in the last place); this is why the oracle has a correctly-rounded mode that
the GPU path is compared with bit for bit."""
import ctypes as C
import os
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("rsqrt") / "librsqrt.so")
    subprocess.run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                    "-I" + os.path.join(ROOT, "melody2d_b200", "csrc"),
                    os.path.join(ROOT, "tests", "emul", "rsqrt_shim.c"), "-o", out, "-lm"], check=True)
    L = C.CDLL(out)
    for f in (L.rsqrt_batch, L.pow_batch):
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        f.restype = None
    return L


def nearest_rsqrt(xs):
    getcontext().prec = 60
    return np.array([float(1 / Decimal(float(x)).sqrt()) for x in xs])


def test_rsqrt_is_correctly_rounded(shim):
    rng = np.random.default_rng(7)
    # squared segment lengths of the workloads span about 1e-14 .. 1e-2 m^2; add wide extremes
    xs = np.concatenate([10.0 ** rng.uniform(-14, 4, 40000), 10.0 ** rng.uniform(-300, 300, 2000)])
    ref = nearest_rsqrt(xs)
    y = np.empty_like(xs)
    shim.rsqrt_batch(xs.ctypes.data, y.ctypes.data, len(xs))
    np.testing.assert_array_equal(y, ref)
    g = np.empty_like(xs)
    shim.pow_batch(xs.ctypes.data, g.ctypes.data, len(xs))
    bad = g != ref
    # glibc's misses are one unit in the last place, never more
    assert np.all(np.abs(g[bad] - ref[bad]) <= np.spacing(ref[bad]))
    print("glibc pow(x,-0.5) misrounded for %d of %d arguments" % (bad.sum(), len(xs)))


def test_rsqrt_special_values(shim):
    xs = np.array([0.0, np.inf, -1.0, np.nan, 4.0, 0.25, 5e-324, 1.7e308])
    y = np.empty_like(xs)
    shim.rsqrt_batch(xs.ctypes.data, y.ctypes.data, len(xs))
    assert y[0] == np.inf and y[1] == 0.0 and np.isnan(y[2]) and np.isnan(y[3])
    assert y[4] == 0.5 and y[5] == 2.0
    assert y[6] == float(1 / Decimal(5e-324).sqrt()) and y[7] == nearest_rsqrt([1.7e308])[0]
