"""GPU parity of the plain FP64 particle filter against the CPU oracle run in
the reference's SMCSampler order (and against the reference's own fixture):
identical resampling decisions and ancestors, ESS history within 1e-12,
log-likelihood within 1e-10 relative; the full-size run is checked against
the Kalman filter's exact log-likelihood."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))
SD0 = 1 / np.sqrt(1 - 0.9 * 0.9)


@pytest.fixture(scope="module")
def env():
    require_cuda()
    import mckl_b200 as mb

    O.build()
    return mb, O.CPUPath("oracle")


def compare(res, want, N):
    assert np.array_equal(res["resampled"], want["resampled"])
    assert np.max(np.abs(res["ess"] - want["ess"]) / want["ess"]) <= 1e-12
    assert abs(res["loglik"] - want["loglik"]) <= 1e-10 * abs(want["loglik"])
    anc = res["anc"].cpu().numpy().astype(np.uint64)
    rows = want["resampled"] == 1
    flips = int(np.sum(anc[rows] != want["anc"][rows]))
    return flips


@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
def test_pf_matches_reference_fixture(env, scheme):
    mb, _ = env
    y = GOLD["pf_y"]
    res = mb.pf_ar1_plain(2000, y, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme=scheme, record=True)
    assert np.array_equal(res["resampled"], GOLD[f"pf_{scheme}_resampled"])
    assert abs(res["loglik"] - GOLD[f"pf_{scheme}_loglik"][0]) <= 1e-10 * abs(GOLD[f"pf_{scheme}_loglik"][0])
    anc = res["anc"].cpu().numpy()[GOLD[f"pf_{scheme}_resampled"] == 1]
    assert np.array_equal(anc.astype(np.uint16), GOLD[f"pf_{scheme}_anc"])
    x = res["x"].cpu().numpy()
    assert np.max(np.abs(x - GOLD[f"pf_{scheme}_x"])) <= 1e-12


@pytest.mark.parametrize("scheme", [2, 1])
def test_pf_vs_oracle(env, scheme):
    mb, orc = env
    _, y = orc.simulate_ar1(60, 0.9, 1.0, 0.5, SD0, (7, 0))
    N = 1 << 14
    want = orc.pf_ar1(N, y, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme)
    res = mb.pf_ar1_plain(N, y, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme=scheme, record=True)
    assert compare(res, want, N) == 0


def test_pf_full_size_against_kalman(env):
    """N = 2^20 particles, T = 1000 observations from seed 7: the log-likelihood
    estimate must be close to the exact Kalman value (Monte Carlo error of a
    2^20-particle filter: a few hundredths), and the first 30 steps must agree
    with the oracle exactly in decisions and ancestors."""
    mb, orc = env
    _, y = orc.simulate_ar1(1000, 0.9, 1.0, 0.5, SD0, (7, 0))
    N = 1 << 20
    kf, _ = orc.kalman_ar1(y, 0.9, 1.0, 0.5)
    res = mb.pf_ar1_plain(N, y, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme=2)
    assert abs(res["loglik"] - kf) < 0.5, (res["loglik"], kf)
    y30 = y[:31]
    want = orc.pf_ar1(N, y30, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), 2)
    res30 = mb.pf_ar1_plain(N, y30, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme=2, record=True)
    assert compare(res30, want, N) == 0


@pytest.mark.parametrize("scheme", [2, 0])
def test_pf_degenerate_weights_vs_oracle(env, scheme):
    """Observation outliers collapse the weights in one step (ESS near 1): the
    resampling then works on cumulative weights with one term just below 1
    and almost all others zero, and a run without resampling (threshold 0)
    drives the weights degenerate over many steps.  Decisions, ancestors,
    ESS and log-likelihood against the oracle, as in the other runs."""
    mb, orc = env
    _, y = orc.simulate_ar1(60, 0.9, 1.0, 0.5, SD0, (8, 0))
    y = y.copy()
    y[12] += 25.0
    y[31] -= 40.0
    y[47] += 15.0
    N = 1 << 14
    want = orc.pf_ar1(N, y, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme)
    res = mb.pf_ar1_plain(N, y, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme=scheme, record=True)
    assert res["resampled"][[12, 31, 47]].all()
    assert compare(res, want, N) == 0
    want0 = orc.pf_ar1(N, y, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme, threshold=0.0)
    res0 = mb.pf_ar1_plain(N, y, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme=scheme, threshold=0.0, record=True)
    assert not res0["resampled"].any()
    assert compare(res0, want0, N) == 0

