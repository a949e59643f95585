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
