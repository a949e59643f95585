"""SMCEstimator's weighted estimate (algorithm/smc.hpp:90-120) on the device:
sum_i W_i u(i, j) in both layouts and every kernel shape (column-major,
row-major with d <= 256 and d > 256), against the oracle's dgemv order and
the exactly rounded sum (math.fsum of the products), within the error bound
of an FP64 sum of n terms; run-to-run bit-identical (fixed summation order)."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402


@pytest.fixture(scope="module")
def mb():
    require_cuda()
    import mckl_b200

    return mckl_b200


@pytest.mark.parametrize("n,d", [(1, 1), (1000, 3), (100000, 4), (8192 * 3 + 5, 2), (20000, 7), (3000, 256),
                                 (2500, 300), (70, 1000)])
def test_weighted_estimate(mb, n, d):
    orc = O.CPUPath("oracle")
    rng = np.random.default_rng(n + d)
    W = rng.random(n)
    W /= W.sum()
    u = rng.normal(size=(n, d)) * 3 + 1
    Wd = torch.from_numpy(W).cuda()
    want = orc.weighted_estimate(u, W)
    for col in (False, True):
        uu = np.ascontiguousarray(u.T if col else u)
        assert np.array_equal(orc.weighted_estimate(uu, W, col_major=col), want)
        ud = torch.from_numpy(uu).cuda()
        got = mb.weighted_estimate(ud, Wd, col_major=col).cpu().numpy()
        again = mb.weighted_estimate(ud, Wd, col_major=col).cpu().numpy()
        assert np.array_equal(got, again)
        for j in range(d):
            exact = math.fsum(W * u[:, j])
            bound = 2 * n * 2.0**-53 * float(np.sum(np.abs(W * u[:, j]))) + 1e-300
            assert abs(got[j] - exact) <= bound, (col, j, got[j], exact)
            assert abs(got[j] - want[j]) <= 2 * bound, (col, j, got[j], want[j])


def test_weighted_estimate_empty(mb):
    out = mb.weighted_estimate(torch.zeros(0, 5, dtype=torch.float64, device="cuda"),
                               torch.zeros(0, dtype=torch.float64, device="cuda"))
    assert out.shape == (5,) and not out.any()
