"""The score estimate by the Fisher identity (mckl_b200_batched_score: PaRIS
smoothing in the batched FP64 filter's forward pass).

* Same forward pass: its log-likelihoods equal the batched FP64 run's bit for
  bit, and two calls give the same scores.
* Consistent: over R = 8 independent runs (model and resampling keys), each
  filter's mean score must lie within 5 Monte Carlo standard errors (plus 2 %
  of the gradient's size, room for the O(1/N) bias of the estimator) of the
  exact Kalman gradient, component by component.
* The fixed-ancestor adjoint of the same runs is a biased estimate of the
  score; the score's error against Kalman must be far below the adjoint's.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    require_cuda()
    import mckl_b200 as mb
    from mckl_b200.kalman import kalman_ar1

    return mb, kalman_ar1


def make(mb, w, threads=512):
    b = mb.BatchedFilters(w["N"], w["y"], w["phi"], w["sx"], w["sy"], w["mkeys"], w["rkeys"], fp64=True)
    b.config(threads, 1)
    return b


def test_score_shares_the_forward_pass(env):
    mb, _ = env
    w = mb.batched_workload(F=10, T=50, seed=71, nmin=300, nmax=5000)
    b = make(mb, w)
    b.run()
    ll, _ = b.results()
    ll2, g = b.score()
    ll3, g2 = b.score()
    b.close()
    assert np.array_equal(ll, ll2) and np.array_equal(ll2, ll3)
    assert np.all(np.isfinite(g)) and np.array_equal(g, g2)


def test_score_converges_to_kalman_gradient(env):
    mb, kalman_ar1 = env
    F, T, N, R = 16, 100, 4096, 8
    w = mb.batched_workload(F=F, T=T, seed=72, nmin=N, nmax=N + 1)
    _, kg = kalman_ar1(w["y"], w["phi"], w["sx"], w["sy"])
    b = make(mb, w)
    S = np.zeros((R, F, 3))
    G = np.zeros((R, F, 3))
    for r in range(R):
        mk = w["mkeys"].copy()
        rk = w["rkeys"].copy()
        mk[:, 1] += 1000 * (r + 1)
        rk[:, 1] += 1000 * (r + 1)
        b.set_keys(mk, rk)
        _, S[r] = b.score()
        _, G[r] = b.adjoint(checkpoint_every=16)
    b.close()
    mean = S.mean(0)
    se = S.std(0, ddof=1) / np.sqrt(R)
    err = np.abs(mean - kg)
    bound = 5.0 * se + 0.02 * np.abs(kg) + 1e-3
    assert np.all(err <= bound), (err.max(), np.argmax(err - bound), (err / bound).max())
    rel_score = np.linalg.norm(mean - kg, axis=1) / np.linalg.norm(kg, axis=1)
    rel_adj = np.linalg.norm(G.mean(0) - kg, axis=1) / np.linalg.norm(kg, axis=1)
    assert np.median(rel_score) < 0.25 * np.median(rel_adj), (np.median(rel_score), np.median(rel_adj))
