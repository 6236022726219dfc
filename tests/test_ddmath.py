"""CPU tests of the correctly rounded log/sin/cos/acos used by the GPU self-block kernel
(best_hydro_b200/csrc/ddmath.cuh), compiled here as host code: each result must equal the
correctly rounded value computed with Python's decimal module at 60 digits, and agree with glibc
(the reference's libm) on all but a rare handful of arguments."""
import ctypes
import math
import os
import subprocess
import tempfile
from decimal import Decimal, getcontext

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
getcontext().prec = 60


@pytest.fixture(scope="module")
def shim():
    d = tempfile.mkdtemp()
    so = os.path.join(d, "ddmath_shim.so")
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=c++17", "-o", so,
                    os.path.join(HERE, "native", "ddmath_shim.cpp")], check=True)
    L = ctypes.CDLL(so)
    dp = ctypes.POINTER(ctypes.c_double)
    for nm in ("dd_log_v", "dd_sin_v", "dd_cos_v", "dd_acos_v"):
        getattr(L, nm).argtypes = [ctypes.c_int, dp, dp]
    L.dd_ln2.argtypes = [dp, dp]
    return L


def call(L, name, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    dp = ctypes.POINTER(ctypes.c_double)
    getattr(L, name)(x.size, x.ctypes.data_as(dp), y.ctypes.data_as(dp))
    return y


def d_pi():
    # Machin: pi = 16 atan(1/5) - 4 atan(1/239)
    def atan_inv(n):
        x = Decimal(1) / n
        x2 = x * x
        s, t, k = Decimal(0), x, 0
        while abs(t) > Decimal(10) ** -70:
            s += t / (2 * k + 1) * (-1) ** k
            t *= x2
            k += 1
        return s
    return 16 * atan_inv(5) - 4 * atan_inv(239)


PI = d_pi()


def d_sincos(x):
    x = Decimal(x)
    s, c = Decimal(0), Decimal(0)
    t = x
    n = 1
    for _ in range(45):  # |x| <= 2 pi: the 45th term is far below 1e-60 relative
        s += t
        t = -t * x * x / ((n + 1) * (n + 2))
        n += 2
    t = Decimal(1)
    n = 0
    for _ in range(45):
        c += t
        t = -t * x * x / ((n + 1) * (n + 2))
        n += 2
    return s, c


def d_acos(x):
    th = Decimal(math.acos(x))
    for _ in range(3):
        s, c = d_sincos(th)
        th = th + (c - Decimal(x)) / s
    return th


def test_pio2_constant_and_ln2(shim):
    a, b, c = Decimal(1.5707963267948966192e+00), Decimal(6.1232339957367660359e-17), Decimal(-1.4973849048591698329e-33)
    assert abs((a + b + c) - PI / 2) < Decimal(10) ** -48
    hi, lo = ctypes.c_double(), ctypes.c_double()
    shim.dd_ln2(ctypes.byref(hi), ctypes.byref(lo))
    assert abs(Decimal(hi.value) + Decimal(lo.value) - Decimal(2).ln()) < Decimal(10) ** -31


def test_log_correctly_rounded(shim):
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(1.0, 50.0, 1500), np.exp(rng.uniform(-30, 30, 500)), [1.0, 2.0, 0.5, 3.0]])
    y = call(shim, "dd_log_v", x)
    want = np.array([float(Decimal(v).ln()) for v in x])
    assert np.array_equal(y, want)
    glibc = np.array([math.log(v) for v in x])
    assert np.count_nonzero(y != glibc) <= 2


def test_sin_cos_correctly_rounded(shim):
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(-math.pi, 2 * math.pi, 1500), rng.uniform(-1e-3, 1e-3, 100),
                        [math.pi, math.pi / 2, 2 * math.pi, 1e-300, 0.0]])
    s = call(shim, "dd_sin_v", x)
    c = call(shim, "dd_cos_v", x)
    ws, wc = zip(*[d_sincos(v) for v in x])
    assert np.array_equal(s, np.array([float(v) for v in ws]))
    assert np.array_equal(c, np.array([float(v) for v in wc]))
    glibc_s = np.array([math.sin(v) for v in x])
    glibc_c = np.array([math.cos(v) for v in x])
    assert np.count_nonzero(s != glibc_s) + np.count_nonzero(c != glibc_c) <= 3


def test_acos_correctly_rounded(shim):
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(-0.999, 0.999, 1000), rng.uniform(0.0, 0.2, 200), [0.5, -0.5, 0.0]])
    y = call(shim, "dd_acos_v", x)
    want = np.array([float(d_acos(v)) for v in x])
    assert np.array_equal(y, want)
    assert np.count_nonzero(y != np.array([math.acos(v) for v in x])) <= 2


def _pairs(L, name, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    hi, lo = np.empty_like(x), np.empty_like(x)
    dp = ctypes.POINTER(ctypes.c_double)
    getattr(L, name)(x.size, x.ctypes.data_as(dp), hi.ctypes.data_as(dp), lo.ctypes.data_as(dp))
    return hi, lo


def _log_samples(n, seed):
    """Arguments that stress the table-driven log: the pair integrals' range (ratios of sums near
    1..2), a wide exponent range, points next to 1 and next to every subinterval boundary."""
    rng = np.random.default_rng(seed)
    near1 = 1.0 + rng.uniform(-2.0 ** -9, 2.0 ** -9, n // 8) * np.exp2(-rng.integers(0, 40, n // 8))
    # bit patterns on both sides of the 256 subinterval boundaries (kLogOff = 0x3FE5F80000000000)
    off = 0x3FE5F80000000000
    b = off + (np.arange(256, dtype=np.uint64) << np.uint64(44))
    bnd = np.concatenate([(b + d).view(np.float64) for d in (np.uint64(0), np.uint64(1))] +
                         [(b - np.uint64(d)).view(np.float64) for d in (1, 2)])
    return np.concatenate([rng.uniform(1.0, 2.0, n // 2), np.exp(rng.uniform(-700, 700, n // 8)),
                           rng.uniform(0.3, 3.0, n // 8), near1, bnd, 2.0 ** np.arange(-1070, 1020, 7.0),
                           [1.0, 2.0, 0.5, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308]])


def test_log_tab_fast_phase_error_bound(shim):
    """The fast phase of cr_log_tab is within 2^-74 of log x (relative), measured against the
    accurate phase (2^-100); its rounding test uses 2^-72."""
    x = _log_samples(400000, 11)
    x = x[(x > 2.3e-308) & (x != 1.0)]
    fh, fl = _pairs(shim, "dd_log_fast_v", x)
    ah, al = _pairs(shim, "dd_log_acc_v", x)
    err = np.abs((fh - ah) + (fl - al)) / np.abs(ah)
    assert float(np.max(err)) < 2.0 ** -74, np.log2(np.max(err))


def test_log_tab_correctly_rounded(shim):
    """cr_log_tab equals the correctly rounded log (Decimal at 60 digits) and cr_log."""
    x = _log_samples(200000, 12)
    y = call(shim, "dd_log_tab_v", x)
    assert np.array_equal(y, call(shim, "dd_log_v", x))
    sub = np.random.default_rng(13).choice(x.size, 3000, replace=False)
    want = np.array([float(Decimal(float(v)).ln()) for v in x[sub]])
    assert np.array_equal(y[sub], want)


def test_log_tab_special_values(shim):
    x = np.array([0.0, -0.0, -1.0, np.inf, np.nan, 1.0, 5e-324])
    y = call(shim, "dd_log_tab_v", x)
    assert y[0] == -np.inf and y[1] == -np.inf and np.isnan(y[2]) and y[3] == np.inf and np.isnan(y[4])
    assert y[5] == 0.0 and not np.signbit(y[5])
    assert y[6] == float(Decimal(5e-324).ln())
