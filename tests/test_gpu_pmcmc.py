"""Particle marginal Metropolis-Hastings over many chains
(mckl_b200_pmcmc_ar1, PMCMCMutation of algorithm/pmcmc.hpp:72-165) against
the same chains run one by one on the CPU: the oracle's particle filter in
the reference's step order, the same keys, the same proposal and acceptance
randomness (Philox4x32 words turned into normals with the C library's
log/cos/sin), and the reference's order of terms in the acceptance test.
With FP64 filters the batched log-likelihoods agree with the oracle's to
~1e-12, so every acceptance decision and every state of every chain agree.
"""
import math

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


def mix32(x):
    x &= 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x85EBCA6B) & 0xFFFFFFFF
    x ^= x >> 13
    x = (x * 0xC2B2AE35) & 0xFFFFFFFF
    x ^= x >> 16
    return x


def philox_words(orc, k0, k1, ctr):
    """Philox4x32-10 block for counter (ctr, 0) from the oracle."""
    e = O.Engine.make(O.PHILOX4X32, key=(k0, k1), ctr=(ctr - 1,) if ctr > 0 else (2**64 - 1,))
    return [int(v) for v in orc.rand(e, 4)]


def log_prior(th):
    phi, sx, sy = th
    if not (0.0 < phi < 1.0 and 0.0 < sx < 5.0 and 0.0 < sy < 5.0):
        return -math.inf
    return -math.log(5.0) * 2  # flat on (0, 1) x (0, 5) x (0, 5)


def random_walk_z(w):
    r0 = math.sqrt(-2.0 * math.log((w[0] + 1.0) * 2.0**-32))
    a0 = 6.283185307179586476925286766559 * (w[1] * 2.0**-32)
    r1 = math.sqrt(-2.0 * math.log((w[2] + 1.0) * 2.0**-32))
    a1 = 6.283185307179586476925286766559 * (w[3] * 2.0**-32)
    return (r0 * math.cos(a0), r0 * math.sin(a0), r1 * math.cos(a1))


def log_scale_walk(step):
    """An asymmetric proposal: phi by a Gaussian step, sx and sy multiplied by
    exp(step z) (a random walk on the log scale), whose log proposal ratio is
    log(sx' / sx) + log(sy' / sy)."""
    def prop(chain, it, w, theta):
        z = random_walk_z(w)
        sx, sy = theta[1], theta[2]
        theta[0] = theta[0] + step[0] * z[0]
        theta[1] = sx * math.exp(step[1] * z[1])
        theta[2] = sy * math.exp(step[2] * z[2])
        return math.log(theta[1] / sx) + math.log(theta[2] / sy)
    return prop


def oracle_pmcmc(orc, y, N, theta0, step, iters, seed, proposal=None):
    C = theta0.shape[0]
    T = y.shape[1] - 1
    th = theta0.copy()
    out = np.zeros((iters, C, 3))
    llo = np.zeros((iters, C))
    acc = np.zeros(C, dtype=np.uint32)

    def pf(c, p, it):
        phi, sx, sy = p
        r = orc.pf_ar1(N, y[c], phi, sx, sy, sx / math.sqrt(1 - phi * phi), (c, mix32(seed ^ (2 * it))),
                       (c, mix32(seed ^ (2 * it + 1))), record=False)
        return r["loglik"]

    ll = np.array([pf(c, th[c], 0) for c in range(C)])
    for it in range(iters):
        if it > 0:
            for c in range(C):
                w = philox_words(orc, seed, c, 2 * it)
                if proposal is None:
                    p = th[c] + step * np.array(random_walk_z(w))
                    lq = 0.0
                else:
                    p = th[c].copy()
                    lq = proposal(c, it, np.array(w, dtype=np.uint32), p)
                inside = p[0] * p[0] < 1 and p[1] > 0 and p[2] > 0
                lp = log_prior(p) if inside else -math.inf
                if not math.isfinite(lp):
                    continue
                llp = pf(c, p, it)
                u = philox_words(orc, seed, c, 2 * it + 1)[0]
                logu = math.log((u + 0.5) * 2.0**-32)
                prob = -log_prior(th[c]) - ll[c]
                prob += lq
                prob += lp
                prob += llp
                if logu < prob:
                    th[c] = p
                    ll[c] = llp
                    acc[c] += 1
        out[it] = th
        llo[it] = ll
    return out, llo, acc


def test_pmcmc_fp64_matches_oracle(env):
    mb, orc = env
    w = mb.batched_workload(F=6, T=40, seed=31, nmin=400, nmax=1200)
    N = 700
    theta0 = np.stack([w["phi"], w["sx"], w["sy"]], axis=1)
    step = np.array([0.02, 0.05, 0.03])
    th, ll, acc = mb.pmcmc_ar1(w["y"], N, theta0, step, log_prior, iters=12, seed=5, fp64=True)
    tho, llo, acco = oracle_pmcmc(orc, w["y"], N, theta0, step, 12, 5)
    assert np.array_equal(acc, acco), (acc, acco)
    assert np.allclose(th, tho, rtol=0, atol=1e-14)
    assert np.allclose(ll, llo, rtol=1e-10, atol=0)
    assert acc.sum() > 0


def test_pmcmc_fp32_chains_move(env):
    mb, orc = env
    w = mb.batched_workload(F=64, T=60, seed=32, nmin=512, nmax=4096)
    theta0 = np.stack([w["phi"], w["sx"], w["sy"]], axis=1)
    th, ll, acc = mb.pmcmc_ar1(w["y"], 1024, theta0, np.array([0.02, 0.05, 0.03]), log_prior, iters=20, seed=9)
    assert th.shape == (20, 64, 3) and np.all(np.isfinite(ll))
    rate = acc.sum() / (64 * 19)
    assert 0.05 < rate < 0.95, rate
    # a chain's state changes exactly at its accepted iterations
    moved = np.any(th[1:] != th[:-1], axis=2).sum(axis=0)
    assert np.array_equal(moved, acc)


def test_pmcmc_proposal_hook_matches_oracle(env):
    """A user proposal (log-scale walk on the scales, asymmetric) through
    mckl_b200_pmcmc_ar1_proposal: every chain equals the CPU loop with the
    same proposal and its log ratio in the acceptance sum."""
    mb, orc = env
    w = mb.batched_workload(F=5, T=40, seed=33, nmin=400, nmax=1200)
    N = 600
    theta0 = np.stack([w["phi"], w["sx"], w["sy"]], axis=1)
    step = np.array([0.02, 0.05, 0.05])
    prop = log_scale_walk(step)
    th, ll, acc = mb.pmcmc_ar1(w["y"], N, theta0, step, log_prior, iters=10, seed=7, fp64=True, proposal=prop)
    tho, llo, acco = oracle_pmcmc(orc, w["y"], N, theta0, step, 10, 7, proposal=prop)
    assert np.array_equal(acc, acco), (acc, acco)
    assert np.allclose(th, tho, rtol=0, atol=1e-14)
    assert np.allclose(ll, llo, rtol=1e-10, atol=0)
    assert acc.sum() > 0


def test_pmcmc_default_equals_explicit_random_walk(env):
    """The built-in random walk and the same walk given as a hook agree."""
    mb, orc = env
    w = mb.batched_workload(F=4, T=30, seed=34, nmin=300, nmax=900)
    theta0 = np.stack([w["phi"], w["sx"], w["sy"]], axis=1)
    step = np.array([0.02, 0.05, 0.03])

    def walk(chain, it, words, theta):
        z = random_walk_z(words)
        for k in range(3):
            theta[k] = theta[k] + step[k] * z[k]
        return 0.0

    a = mb.pmcmc_ar1(w["y"], 500, theta0, step, log_prior, iters=8, seed=3, fp64=True)
    b = mb.pmcmc_ar1(w["y"], 500, theta0, step, log_prior, iters=8, seed=3, fp64=True, proposal=walk)
    assert np.array_equal(a[2], b[2])
    assert np.allclose(a[0], b[0], rtol=0, atol=1e-14) and np.array_equal(a[1], b[1])
