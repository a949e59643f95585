"""GPU parity of the plain FP64 particle filter at its full configuration:
AR(1) with phi 0.9, sx 1, sy 0.5, T = 1000 observations simulated from seed 7,
N = 2^20 particles, resampling when ESS < N/2 with each of the multinomial,
stratified, systematic and residual schemes.

The fixture (tests/golden/c3_full.npz, made by
``python tests/golden/make_golden.py --c3``) holds the compiled reference's
SMCSampler + BackendSEQ run: every iteration's resampling decision, two exact
integer sums of every parent vector (sum idx_i and sum idx_i (i + 1), which
move if any parent changes), the ESS history and the log-likelihood.  The
GPU run must reproduce every decision and every parent-vector digest of all
1000 steps; its ESS history within 1e-12 and its log-likelihood within 1e-10
relative.  A flipped ancestor (a uniform within an ulp of a cumulative weight
whose fold differs by an ulp) would change every later digest: the test
reports the first differing step and the tie count of the run.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

C3 = np.load(os.path.join(os.path.dirname(__file__), "golden", "c3_full.npz"))
SD0 = 1 / np.sqrt(1 - 0.9 * 0.9)


@pytest.fixture(scope="module")
def mb():
    require_cuda()
    import mckl_b200

    return mckl_b200


def digests(anc, rows, chunk=64):
    """(sum idx_i, sum idx_i (i + 1)) of the parent vectors in `rows` of the
    device matrix anc [T + 1, N] (exact in int64 below 2^31 particles)."""
    N = anc.shape[1]
    w = torch.arange(1, N + 1, dtype=torch.int64, device=anc.device)
    out = np.zeros((anc.shape[0], 2), dtype=np.uint64)
    idx = np.flatnonzero(rows)
    for k in range(0, len(idx), chunk):
        r = torch.from_numpy(idx[k:k + chunk]).to(anc.device)
        a = anc.index_select(0, r)
        d1 = a.sum(1)
        d2 = (a * w).sum(1)
        out[idx[k:k + chunk], 0] = d1.cpu().numpy().astype(np.uint64)
        out[idx[k:k + chunk], 1] = d2.cpu().numpy().astype(np.uint64)
    return out


@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
def test_plain_filter_full_config_vs_reference(mb, scheme):
    y = C3["y"]
    N = int(C3["N"][0])
    res = mb.pf_ar1_plain(N, y, 0.9, 1.0, 0.5, SD0, (11, 0), (12, 0), scheme=scheme, record=True)
    want_rs = C3[f"s{scheme}_resampled"]
    assert np.array_equal(res["resampled"], want_rs), \
        ("resampling decisions differ", np.flatnonzero(res["resampled"] != want_rs)[:5])
    rows = want_rs == 1
    got = digests(res["anc"], rows)
    want = C3[f"s{scheme}_digest"]
    bad = np.flatnonzero(np.any(got[rows] != want[rows], axis=1))
    steps = np.flatnonzero(rows)
    ties = res.get("ties")
    assert bad.size == 0, (f"scheme {scheme}: parent vectors differ from the reference from step "
                           f"{steps[bad[0]]} on ({bad.size} of {rows.sum()} resampling steps); ties: {ties}")
    assert np.max(np.abs(res["ess"] - C3[f"s{scheme}_ess"]) / C3[f"s{scheme}_ess"]) <= 1e-12
    ll = float(C3[f"s{scheme}_loglik"][0])
    assert abs(res["loglik"] - ll) <= 1e-10 * abs(ll), (res["loglik"], ll)
    x = res["x"].cpu().numpy()
    xs = C3[f"s{scheme}_x"]
    assert abs(x.sum() - xs[0]) <= 1e-9 * np.abs(x).sum() and x.min() == pytest.approx(xs[1], rel=1e-12) \
        and x.max() == pytest.approx(xs[2], rel=1e-12)
    del res
    torch.cuda.empty_cache()
