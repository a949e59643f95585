"""The library's double-double log / exp / sin / cos on the device against the
C library the reference's transforms call (through the oracle).  They must
agree to within 1 ULP everywhere and exactly in all but a small fraction of
arguments (the C library's own misrounded cases)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402


@pytest.fixture(scope="module")
def env():
    require_cuda()
    import mckl_b200 as mb

    O.build()
    return mb, O.CPUPath("oracle")


def ulps(a, b):
    d = np.abs(a - b)
    return np.where(d == 0, 0.0, d / np.spacing(np.maximum(np.abs(a), np.abs(b))))


def check(got, want, max_mismatch):
    u = ulps(got, want)
    assert u.max() <= 1.0
    assert np.mean(u > 0) <= max_mismatch


def test_log(env):
    mb, orc = env
    rng = np.random.default_rng(1)
    u = (rng.integers(0, 2**32, 1 << 20, dtype=np.uint64).astype(np.float64) + 1) * 2.0**-32
    wide = np.exp(rng.uniform(-700, 700, 1 << 18))
    edge = np.array([1.0, 0.5, 2.0, 5e-324, 2.2250738585072014e-308, 1e-310, np.sqrt(0.5), np.sqrt(2.0)])
    for x in (u, wide, edge):
        got = mb.math_f64("log", torch.from_numpy(x).cuda()).cpu().numpy()
        check(got, orc.math_f64("log", x), 0.005)


def test_exp(env):
    mb, orc = env
    rng = np.random.default_rng(2)
    for x in (rng.uniform(-40, 0, 1 << 20), rng.uniform(-700, 700, 1 << 18),
              np.array([0.0, -0.0, 1e-20, -1e-20, 0.5, -0.5, 709.0, -700.0])):
        got = mb.math_f64("exp", torch.from_numpy(x).cuda()).cpu().numpy()
        check(got, orc.math_f64("exp", x), 0.005)


def test_sincos(env):
    mb, orc = env
    rng = np.random.default_rng(3)
    v = (rng.integers(0, 2**32, 1 << 20, dtype=np.uint64).astype(np.float64) + 1) * 2.0**-32
    for x in (float.fromhex("0x1.921fb54442d18p+2") * v, rng.uniform(-1e4, 1e4, 1 << 18),
              np.array([0.0, np.pi / 4, np.pi / 2, np.pi, 2 * np.pi, 1e-300])):
        s, c = mb.math_f64("sincos", torch.from_numpy(x).cuda())
        ws, wc = orc.math_f64("sincos", x)
        check(s.cpu().numpy(), ws, 0.01)
        check(c.cpu().numpy(), wc, 0.01)
