"""The device math of crmath.cuh (double-double log and exp, rounded once)
compiled for the host from the same source, against exactly computed values
(Python's decimal module at 60 digits): all within one ULP of the exact value,
and the correctly rounded double in all but a few cases per million.  The GPU
tests check the device build against the C library the reference calls."""
import ctypes
import os
import subprocess
import tempfile
from decimal import Decimal, getcontext

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "mckl_b200", "csrc")

SRC = r"""
#include "crmath.cuh"
extern "C" void cr_log(long n, const double *x, double *y) { for (long i = 0; i < n; ++i) y[i] = mckl_b200::dd::log(x[i]); }
extern "C" void cr_exp(long n, const double *x, double *y) { for (long i = 0; i < n; ++i) y[i] = mckl_b200::dd::exp(x[i]); }
extern "C" void cr_exp_dd(long n, const double *x, double *y) { for (long i = 0; i < n; ++i) y[i] = mckl_b200::dd::exp_dd(x[i]); }
extern "C" void cr_sincos(long n, const double *x, double *s, double *c) { for (long i = 0; i < n; ++i) mckl_b200::dd::sincos(x[i], s + i, c + i); }
extern "C" void cr_sincos_dd(long n, const double *x, double *s, double *c) { for (long i = 0; i < n; ++i) mckl_b200::dd::sincos_dd(x[i], s + i, c + i); }
extern "C" long cr_sincos_quick(long n, const double *x, double *s, double *c) {
    long ok = 0;
    for (long i = 0; i < n; ++i) { if (mckl_b200::dd::sincos_quick(x[i], s + i, c + i)) ++ok; else s[i] = c[i] = 9.0; }
    return ok;
}
extern "C" long cr_exp_quick(long n, const double *x, double *y) {
    long ok = 0;
    for (long i = 0; i < n; ++i) { double v = 0; if (mckl_b200::dd::exp_quick(x[i], &v)) { ++ok; y[i] = v; } else y[i] = -1.0; }
    return ok;
}
"""


@pytest.fixture(scope="module")
def lib():
    d = tempfile.mkdtemp()
    src, so = os.path.join(d, "cr.cpp"), os.path.join(d, "libcr.so")
    with open(src, "w") as f:
        f.write(SRC)
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I", CSRC, src,
                        "-o", so], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("host compiler unavailable: " + r.stderr[:200])
    return ctypes.CDLL(so)


def run(lib, name, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    getattr(lib, name)(ctypes.c_long(len(x)), x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p))
    return y


def exact_check(xs, ys, fn):
    getcontext().prec = 60
    off = 0
    for x, y in zip(xs, ys):
        e = fn(Decimal(float(x)))
        rn = float(e)  # correctly rounded (round-half-even of the 60-digit value)
        if y != rn:
            off += 1
            assert abs(Decimal(float(y)) - e) <= Decimal(float(np.spacing(abs(rn)))), (x, y, rn)
    return off


def test_log_correctly_rounded(lib):
    rng = np.random.default_rng(11)
    u = (rng.integers(0, 2**32, 40000).astype(np.float64) + 0.5) * 2.0**-32   # U01OO of u32 words
    w = np.exp(rng.uniform(-700, 700, 20000))
    near1 = 1.0 + rng.integers(-2**20, 2**20, 20000) * 2.0**-52
    xs = np.concatenate([u, w, near1[near1 > 0], [1.0, 2.0, 0.5, 5e-324, 2.2250738585072014e-308]])
    off = exact_check(xs, run(lib, "cr_log", xs), lambda d: d.ln())
    assert off <= 2, off


def test_exp_correctly_rounded(lib):
    rng = np.random.default_rng(12)
    xs = np.concatenate([rng.uniform(-40, 0, 40000), rng.uniform(-700, 700, 20000), [0.0, 1e-20, -1e-20, 0.5]])
    off = exact_check(xs, run(lib, "cr_exp", xs), lambda d: d.exp())
    assert off <= 2, off


def test_exp_quick_phase_equals_accurate_phase(lib):
    """The quick phase (Tang's table method with Ziv's rounding test) returns
    only values the accurate double-double phase also returns: identical bits
    on a million arguments over the weight normaliser's range (log-weights
    minus their maximum), the whole normal range, near 0 and near the
    table's and the binades' edges; and it settles all but a few in a
    thousand."""
    rng = np.random.default_rng(13)
    ln2_64 = np.log(2.0) / 64
    xs = np.concatenate([
        rng.uniform(-40, 0, 400000),
        rng.uniform(-708, 709, 300000),
        rng.uniform(-1e-3, 1e-3, 100000),
        # around k ln2/64 +- ln2/128 (the reduction's edges) and k ln2 (binade edges of the result)
        (rng.integers(-65000, 65000, 100000) + rng.choice([-0.5, 0.5, 0.0], 100000)) * ln2_64
        + rng.uniform(-1e-12, 1e-12, 100000),
        rng.integers(-1000, 1000, 100000) * np.log(2.0) + rng.uniform(-1e-9, 1e-9, 100000),
    ])
    xs = xs[(xs >= -745) & (xs <= 709.7)]
    full = run(lib, "cr_exp", xs)
    acc = run(lib, "cr_exp_dd", xs)
    assert np.array_equal(full.view(np.int64), acc.view(np.int64))
    xs_q = np.ascontiguousarray(xs)
    yq = np.empty_like(xs_q)
    lib.cr_exp_quick.restype = ctypes.c_long
    ok = lib.cr_exp_quick(ctypes.c_long(len(xs_q)), xs_q.ctypes.data_as(ctypes.c_void_p),
                          yq.ctypes.data_as(ctypes.c_void_p))
    taken = yq != -1.0
    assert np.array_equal(yq[taken].view(np.int64), acc[taken].view(np.int64))
    assert ok == taken.sum() and ok >= 0.99 * len(xs_q), ok / len(xs_q)


def _sincos(lib, name, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    sn, cs = np.empty_like(x), np.empty_like(x)
    fn = getattr(lib, name)
    fn.restype = ctypes.c_long
    n = fn(ctypes.c_long(len(x)), x.ctypes.data_as(ctypes.c_void_p), sn.ctypes.data_as(ctypes.c_void_p),
           cs.ctypes.data_as(ctypes.c_void_p))
    return sn, cs, n


def test_sincos_quick_phase_equals_accurate_phase(lib):
    """The quick phase of sincos (table of sin, cos at j/64, angle addition,
    Ziv's test) returns only values the accurate phase also returns: the
    Box-Muller angles 2 pi v of U01 words, the transforms' whole range below
    1e5, arguments near multiples of pi/2 and pi/4, tiny ones; and it settles
    all but a few in a thousand."""
    rng = np.random.default_rng(14)
    u = (rng.integers(0, 2**32, 400000).astype(np.float64) + 0.5) * 2.0**-32
    xs = np.concatenate([
        2 * np.pi * u,
        rng.uniform(-1e5, 1e5, 200000),
        rng.integers(-60000, 60000, 100000) * (np.pi / 2) + rng.uniform(-1e-6, 1e-6, 100000),
        rng.integers(-100, 100, 100000) * (np.pi / 4) + rng.uniform(-1e-12, 1e-12, 100000),
        rng.uniform(-1e-8, 1e-8, 50000), rng.integers(-64, 64, 50000) / 64.0 + rng.uniform(-1e-3, 1e-3, 50000),
    ])
    s1, c1, _ = _sincos(lib, "cr_sincos", xs)
    s2, c2, _ = _sincos(lib, "cr_sincos_dd", xs)
    assert np.array_equal(s1.view(np.int64), s2.view(np.int64))
    assert np.array_equal(c1.view(np.int64), c2.view(np.int64))
    sq, cq, ok = _sincos(lib, "cr_sincos_quick", xs)
    taken = sq != 9.0
    assert np.array_equal(sq[taken].view(np.int64), s2[taken].view(np.int64))
    assert np.array_equal(cq[taken].view(np.int64), c2[taken].view(np.int64))
    assert ok == taken.sum() and ok >= 0.99 * len(xs), ok / len(xs)


def test_sincos_correctly_rounded(lib):
    """sin and cos of the Box-Muller angles and of the whole range against
    the exactly computed values (60 digits): all within one ULP, the correctly
    rounded double in all but a few cases."""
    rng = np.random.default_rng(15)
    u = (rng.integers(0, 2**32, 6000).astype(np.float64) + 0.5) * 2.0**-32
    xs = np.concatenate([2 * np.pi * u, rng.uniform(-1e4, 1e4, 2000)])
    sn, cs, _ = _sincos(lib, "cr_sincos", xs)
    getcontext().prec = 60

    def dsin(d):
        # reduce by 2 pi at 60 digits, then the Taylor series
        pi = Decimal("3.14159265358979323846264338327950288419716939937510582097494459")
        d = d % (2 * pi)
        s, term, n = Decimal(0), d, 1
        while abs(term) > Decimal(10) ** -70:
            s += term
            term = -term * d * d / ((n + 1) * (n + 2))
            n += 2
        return s

    def dcos(d):
        pi = Decimal("3.14159265358979323846264338327950288419716939937510582097494459")
        return dsin(d + pi / 2)

    assert exact_check(xs, sn, dsin) <= 2
    assert exact_check(xs, cs, dcos) <= 2

