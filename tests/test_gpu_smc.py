"""GPU parity of the SMC step: the exact sequential fold, Weight
normalisation, the six resampling schemes, rep -> index and select, against
the CPU oracle and the fixtures produced by the reference itself.

Bars:
  * fold: every partial sum bit-identical to the sequential loop;
  * replication counts, parent indices, engine state: bit-identical;
  * Weight: the normalised weights within 2 ULP (exp/log are rounded
    correctly on the device and nearly always by the C library), ESS and
    log normaliser within 1e-13 relative.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


@pytest.fixture(scope="module")
def env():
    require_cuda()
    import mckl_b200 as mb

    O.build()
    return mb, O.CPUPath("oracle")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def fold_inputs():
    rng = np.random.default_rng(7)
    out = []
    for n in (1, 2, 5, 4095, 4096, 4097, 12289, 1 << 20):
        w = rng.random(n)
        out.append(("uniform", w / w.sum()))
        out.append(("raw", rng.random(n) * 3.0))
    n = 1 << 18
    out.append(("lognormal", np.exp(rng.normal(0, 4, n))))
    z = rng.random(n)
    z[rng.random(n) < 0.3] = 0.0
    out.append(("zeros", z))
    out.append(("equal", np.full(300000, 1.0 / 300000)))
    out.append(("pow2", np.full(100000, 2.0**-17)))       # exact sums, no rounding at all
    out.append(("ties", np.full(50000, 1.0 + 2.0**-52)))   # increments that tie at coarser grids
    out.append(("tiny", np.full(20000, 5e-324)))
    big = rng.random(70000)
    big[::7000] = 1e6
    out.append(("spikes", big))
    # leading zeros (a zero running sum is exact): degenerate weights, a
    # run of zeros before the first positive value, zeros then subnormals
    lead = rng.random(300000)
    lead[:250000] = 0.0
    out.append(("leading zeros", lead))
    deg = np.zeros(1 << 20)
    hit = rng.integers(0, 1 << 20, 40)
    deg[hit] = np.exp(rng.normal(0, 30, 40))
    deg[hit[:5]] = 5e-324 * rng.integers(1, 1000, 5)
    out.append(("degenerate", deg))
    sub = np.zeros(60000)
    sub[20000:] = 5e-324 * rng.integers(0, 4, 40000)
    out.append(("zeros then subnormals", sub))
    out.append(("all zeros", np.zeros(10000)))
    # a subnormal running sum followed by zeros and small values, crossing
    # into the normal range (every sum below 2^-1021 is exact)
    sn = np.zeros(200000)
    sn[1000] = 3e-320
    sn[rng.integers(2000, 200000, 300)] = 5e-324 * rng.integers(1, 2**40, 300)
    sn[150000] = 1e-300
    out.append(("subnormal sums", sn))
    # normalised degenerate weights: one weight just below 1, a few tiny
    # ones, zeros elsewhere (the cumulative sums stay just below 1)
    nd = np.zeros(1 << 20)
    pos = rng.integers(0, 1 << 20, 600)
    nd[pos] = np.exp(rng.normal(-40, 8, 600))
    nd[pos[0]] = 1.0
    out.append(("normalised degenerate", nd * (1.0 / np.cumsum(nd)[-1])))
    # more windows than the list holds: 1 + 2^-53 is a tie (it rounds back to
    # 1), so every element after the first is a window and the fold takes
    # the event loop; appended ordinary values give that loop certain tiles
    # whose descriptors come from the counting pass
    tie = np.concatenate([[1.0], np.full(20000, 2.0**-53)])
    out.append(("ties everywhere", tie))
    out.append(("ties then values", np.concatenate([tie, rng.random(280000)])))
    return out


def test_fold_exact(env):
    mb, orc = env
    for name, x in fold_inputs():
        want_pre, want_fin = orc.fold(x)
        pre, fin = mb.fold_f64(dev(x))
        got = pre.cpu().numpy()
        bad = np.flatnonzero(got.view(np.uint64) != want_pre.view(np.uint64))
        assert bad.size == 0, (name, len(x), bad[:5], got[bad[:3]], want_pre[bad[:3]])
        assert fin == want_fin, name


def test_fold_with_start_value(env):
    mb, orc = env
    x = np.random.default_rng(3).random(50000)
    for s0 in (0.5, 1e10, 3.0):
        want_pre, want_fin = orc.fold(x, s0)
        pre, fin = mb.fold_f64(dev(x), s0)
        assert np.array_equal(pre.cpu().numpy(), want_pre) and fin == want_fin


def ulps(a, b):
    d = np.abs(a - b)
    return np.where(d == 0, 0.0, d / np.spacing(np.maximum(np.abs(a), np.abs(b))))


@pytest.mark.parametrize("N", [1, 7, 1023, 1024, 1025, 5000, 1 << 20])
def test_weight_set_and_add_log(env, N):
    mb, orc = env
    rng = np.random.default_rng(N)
    v = rng.normal(0, 5, N)
    W0, ess0 = orc.weight_set_log(v)
    w = mb.Weight(N)
    w.set_log(dev(v))
    got = w.data.cpu().numpy()
    assert ulps(got, W0).max() <= 2
    assert abs(w.ess() - ess0) <= 1e-13 * ess0
    v2 = rng.normal(0, 2, N)
    W1, ess1 = orc.weight_add_log(W0, v2)
    w.data.copy_(dev(W0))
    w.add_log(dev(v2))
    got = w.data.cpu().numpy()
    assert ulps(got, W1).max() <= 2
    assert abs(w.ess() - ess1) <= 1e-13 * ess1
    # log normaliser increment: log sum_i W0_i exp(v2_i)
    m = v2.max()
    want = m + np.log(np.sum(W0 * np.exp(v2 - m)))
    assert abs(w.log_nc - want) <= 1e-12 * max(1.0, abs(want))


def test_weight_matches_reference_fixture(env):
    mb, _ = env
    w = mb.Weight(5000)
    w.set_log(dev(GOLD["weight_v"]))
    assert ulps(w.data.cpu().numpy(), GOLD["weight_W"]).max() <= 2
    w.data.copy_(dev(GOLD["weight_W"]))
    w.add_log(dev(GOLD["weight_v2"]))
    assert ulps(w.data.cpu().numpy(), GOLD["weight_W2"]).max() <= 2
    assert abs(w.ess() - GOLD["weight_ess2"][0]) <= 1e-13 * GOLD["weight_ess2"][0]


def engines(mb, key=(9,)):
    g = mb.Philox4x32()
    g.key = key
    e = O.Engine.make(1, key=key)
    return g, e


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_u01_sequences(env, kind):
    mb, orc = env
    for n in (0, 1, 1023, 1024, 1025, 5000, 1 << 18):
        g, e = engines(mb)
        got = mb.u01_sequence(kind, g, n).cpu().numpy()
        want = orc.u01_sequence(kind, e, n)
        assert g.state_tuple() == e.state(), (kind, n)
        if n == 0:
            assert got.size == 0
        elif kind == 0:
            # u = 1 - exp(lmax): a cancellation, so the error scale is ulp(1)
            assert np.abs(got - want).max() <= np.spacing(1.0) and np.mean(got != want) < 0.01
        else:
            assert np.array_equal(got, want), (kind, n)


@pytest.mark.parametrize("scheme", range(6))
def test_resample_matches_reference_fixture(env, scheme):
    mb, _ = env
    W = dev(GOLD["weight_W2"])
    for M in (5000, 3333, 7777):
        g, e = engines(mb)
        rep = mb.resample(scheme, g, W, M)
        got = rep.cpu().numpy().astype(np.uint64)
        assert np.array_equal(got, GOLD[f"rs_{scheme}_{M}_rep"]), (scheme, M)
        st = np.array(list(g.state.ctr) + list(g.state.key) + list(g.state.tweak) + [g.state.index, g.state.kind],
                      dtype=np.uint64)
        assert np.array_equal(st, GOLD[f"rs_{scheme}_{M}_state"])
        idx = mb.rep_to_index(rep, M).cpu().numpy().astype(np.uint64)
        assert np.array_equal(idx, GOLD[f"rs_{scheme}_{M}_idx"]), (scheme, M)


@pytest.mark.parametrize("scheme", range(6))
def test_resample_large(env, scheme):
    mb, orc = env
    rng = np.random.default_rng(100 + scheme)
    for N, M in ((1 << 20, 1 << 20), (300001, 123457), (1, 10), (10, 1), (2, 0)):
        W = np.exp(rng.normal(0, 3, N))
        W /= W.sum()
        g, e = engines(mb, key=(scheme + 1, 2))
        rep = mb.resample(scheme, g, dev(W), M)
        want = orc.resample(scheme, e, W, M)
        got = rep.cpu().numpy().astype(np.uint64)
        assert np.array_equal(got, want), (scheme, N, M, np.flatnonzero(got != want)[:5])
        assert g.state_tuple() == e.state()
        if M > 0:
            idx = mb.rep_to_index(rep, M).cpu().numpy().astype(np.uint64)
            assert np.array_equal(idx, orc.rep_index(want, M))


def test_rep_to_index_edge_cases(env):
    mb, orc = env
    cases = [np.array([5, 0, 0, 0, 0]), np.array([0, 0, 0, 0, 5]), np.array([1, 1, 1]), np.array([3]),
             np.array([0, 2, 0, 2, 0, 1]), np.array([0, 0, 7]), np.array([7, 0, 0])]
    for rep in cases:
        for M in (int(rep.sum()),):
            idx = mb.rep_to_index(dev(rep.astype(np.int64)), M).cpu().numpy().astype(np.uint64)
            assert np.array_equal(idx, orc.rep_index(rep.astype(np.uint64), M)), rep


def test_select(env):
    mb, orc = env
    rng = np.random.default_rng(9)
    N = 100000
    W = rng.random(N)
    W /= W.sum()
    rep = orc.resample(2, O.Engine.make(1, key=(4,)), W)
    idx = orc.rep_index(rep)
    st = rng.normal(size=(N, 3))
    want = orc.select_f64(idx, st)
    x = dev(np.ascontiguousarray(st.T))  # dim-major [3, N] == column-major N x 3
    mb.select(dev(idx.astype(np.int64)), x)
    assert np.array_equal(x.cpu().numpy().T, want)
    xf = dev(np.ascontiguousarray(st[:, 0].astype(np.float32)))
    mb.select(dev(idx.astype(np.int64)), xf)
    assert np.array_equal(xf.cpu().numpy(), st[:, 0].astype(np.float32)[idx.astype(np.int64)])
