"""The adjoint of the batched FP64 filters (mckl_b200_batched_adjoint) and its
torch.autograd binding.

* Same estimate: the adjoint's forward pass is the batched FP64 kernel's step,
  so its log-likelihoods equal the batched FP64 run's bit for bit.
* Same function as finite differences: central differences with h = 1e-5
  under common random numbers and the base run's ancestors (the FP64 shadow
  at theta +- h follows the base run's decisions) -- relative error <= 1e-4
  against max(|FD|, 1), the same bar as the gradient target.
* The checkpoint interval changes nothing: the replay reproduces the forward
  pass exactly, so gradients with different intervals are identical.
* Kalman: with the ancestors frozen the gradient ignores how the resampling
  moves with theta, so it is a biased estimate of the exact score at any N;
  it is checked for direction and size against the Kalman gradient (the
  1e-4 bar applies to the function it differentiates, checked by FD).
"""
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


@pytest.fixture(scope="module")
def small(env):
    mb, _ = env
    w = mb.batched_workload(F=12, T=60, seed=99, nmin=300, nmax=3000)
    w["threads"] = 256
    return w


def make(mb, w, **kw):
    b = mb.BatchedFilters(w["N"], w["y"], w["phi"], w["sx"], w["sy"], w["mkeys"], w["rkeys"], **kw)
    b.config(w["threads"], 1)
    return b


def test_adjoint_loglik_matches_batched_fp64(env, small):
    mb, _ = env
    b = make(mb, small, fp64=True)
    b.run()
    ll, _ = b.results()
    ll2, g = b.adjoint(checkpoint_every=7)
    b.close()
    assert np.array_equal(ll, ll2)
    assert np.all(np.isfinite(g))


def test_adjoint_vs_finite_differences(env, small):
    mb, _ = env
    from mckl_b200 import autograd as AG

    b = make(mb, small, fp64=True)
    _, g = b.adjoint(checkpoint_every=16)
    b.close()
    fd = AG.finite_differences(small, h=1e-5, threads=small["threads"])
    rel = np.abs(g - fd) / np.maximum(np.abs(fd), 1.0)
    assert rel.max() <= 1e-4, (rel.max(), g, fd)


def test_adjoint_checkpoint_interval_invariance(env, small):
    mb, _ = env
    b = make(mb, small, fp64=True)
    _, g1 = b.adjoint(checkpoint_every=1)
    _, g2 = b.adjoint(checkpoint_every=13)
    _, g3 = b.adjoint(checkpoint_every=1000)  # one block: T < interval
    b.close()
    assert np.array_equal(g1, g2) and np.array_equal(g1, g3)


def test_autograd_function(env, small):
    mb, orc = env
    from mckl_b200 import autograd as AG

    phi = torch.tensor(small["phi"], requires_grad=True)
    sx = torch.tensor(small["sx"], requires_grad=True)
    sy = torch.tensor(small["sy"], requires_grad=True)
    ll = AG.loglik(phi, sx, sy, small, 16)
    ll.sum().backward()
    b = make(mb, small, fp64=True)
    ll2, g = b.adjoint(16)
    b.close()
    assert np.array_equal(ll.detach().numpy(), ll2)
    assert np.array_equal(phi.grad.numpy(), g[:, 0])
    assert np.array_equal(sx.grad.numpy(), g[:, 1])
    assert np.array_equal(sy.grad.numpy(), g[:, 2])


def test_adjoint_vs_kalman_gradient(env):
    """Large N: the fixed-ancestor gradient against the exact score.  Freezing
    the ancestors drops the dependence of the resampling on theta, so this
    gradient is a biased estimate of the score whatever N is (it drops the
    score of the resampling step); the check is only that it points into the
    same half-space as the exact score with a bias of the order of its size,
    and that the log-likelihood itself is close to Kalman's.  Measured here
    (8 sets, T = 100): cosine 0.73, relative error of the vector 1.43; the
    bars are cosine above 0.6 and relative error below 2.  (At the
    differentiated configuration, 256 sets x T = 1000, the bench measures a
    median cosine of 0.94 and a median relative error of 0.95.)  The
    consistent estimate of the score, and its error against Kalman within its
    Monte Carlo error, is test_gpu_score's; the benchmark reports both."""
    mb, orc = env
    w = mb.batched_workload(F=8, T=100, seed=5, nmin=1 << 16, nmax=(1 << 16) + 1)
    w["threads"] = 512
    b = make(mb, w, fp64=True)
    ll, g = b.adjoint(checkpoint_every=32)
    b.close()
    kg = np.zeros_like(g)
    for f in range(len(ll)):
        kll, kg[f] = orc.kalman_ar1(w["y"][f], w["phi"][f], w["sx"][f], w["sy"][f])
        assert abs(ll[f] - kll) < 1.0, (f, ll[f], kll)
    cos = float(np.sum(g * kg) / (np.linalg.norm(g) * np.linalg.norm(kg)))
    rel = float(np.linalg.norm(g - kg) / np.linalg.norm(kg))
    assert cos > 0.6 and rel < 2.0, (cos, rel)
