"""Pin the CPU oracle (oracle/oracle.c) to the reference.

1. Against the committed golden fixtures (tests/golden/golden.npz, produced by
   the reference compiled from its own headers; see make_golden.py).
2. Against the reference's own known-answer files when the reference source
   tree is present.
3. Against the compiled reference (oracle/_ref) on extra randomized cases
   when that library has been built.
"""
import os

import numpy as np
import pytest

import oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


@pytest.fixture(scope="module")
def orc():
    O.build()
    return O.CPUPath("oracle")


def state_arr(e):
    return np.array(list(e.ctr) + list(e.key) + list(e.tweak) + [e.index, e.kind], dtype=np.uint64)


def same_bits(a, b):
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("kind", range(1, 7))
def test_rand_streams(orc, kind):
    for seed in (1, 42):
        e = O.Engine.make(kind, key=(seed,))
        w = orc.rand(e, 1000)
        assert same_bits(w, GOLD[f"rand_{kind}_{seed}"])
        assert np.array_equal(state_arr(e), GOLD[f"rand_{kind}_{seed}_state"])
    e = O.Engine.make(kind, key=(42, 7), ctr=(2**64 - 3, 5), index=1)
    assert same_bits(orc.rand(e, 777), GOLD[f"rand_{kind}_carry"])
    assert np.array_equal(state_arr(e), GOLD[f"rand_{kind}_carry_state"])


@pytest.mark.parametrize("kind", (1, 3, 5, 2))
def test_u01(orc, kind):
    for var in O.U01_VARIANTS:
        for f64 in (False, True):
            e = O.Engine.make(kind, key=(42,), ctr=(3,), index=1)
            assert same_bits(orc.u01(e, var, f64, 1501), GOLD[f"u01_{kind}_{var}_{int(f64)}"]), (var, f64)
            assert np.array_equal(state_arr(e), GOLD[f"u01_{kind}_{var}_{int(f64)}_state"])


@pytest.mark.parametrize("kind", (1, 3, 5, 2))
def test_normal_exponential_gamma(orc, kind):
    for f64 in (False, True):
        for (mean, sd) in ((0.0, 1.0), (1.5, 2.0)):
            e = O.Engine.make(kind, key=(42,))
            assert same_bits(orc.normal(e, f64, 4097, mean, sd), GOLD[f"normal_{kind}_{int(f64)}_{mean}"])
            assert np.array_equal(state_arr(e), GOLD[f"normal_{kind}_{int(f64)}_{mean}_state"])
        e = O.Engine.make(kind, key=(42,))
        assert same_bits(orc.exponential(e, f64, 5000, 2.0), GOLD[f"exp_{kind}_{int(f64)}"])
        assert np.array_equal(state_arr(e), GOLD[f"exp_{kind}_{int(f64)}_state"])
        for alpha in (0.3, 0.7, 1.0, 2.5, 9.7):
            e = O.Engine.make(kind, key=(42,))
            assert same_bits(orc.gamma(e, f64, 4096, alpha, 1.0), GOLD[f"gamma_{kind}_{int(f64)}_{alpha}"])
            assert np.array_equal(state_arr(e), GOLD[f"gamma_{kind}_{int(f64)}_{alpha}_state"])


def test_weight(orc):
    W, ess = orc.weight_set_log(GOLD["weight_v"])
    assert same_bits(W, GOLD["weight_W"]) and ess == GOLD["weight_ess"][0]
    W2, ess2 = orc.weight_add_log(W, GOLD["weight_v2"])
    assert same_bits(W2, GOLD["weight_W2"]) and ess2 == GOLD["weight_ess2"][0]


@pytest.mark.parametrize("scheme", range(6))
def test_resample(orc, scheme):
    for M in (5000, 3333, 7777):
        e = O.Engine.make(1, key=(9,))
        rep = orc.resample(scheme, e, GOLD["weight_W2"], M)
        assert np.array_equal(rep, GOLD[f"rs_{scheme}_{M}_rep"])
        assert np.array_equal(orc.rep_index(rep, M), GOLD[f"rs_{scheme}_{M}_idx"])
        assert np.array_equal(state_arr(e), GOLD[f"rs_{scheme}_{M}_state"])


@pytest.mark.parametrize("scheme", (0, 1, 2, 3))
def test_particle_filter(orc, scheme):
    y = GOLD["pf_y"]
    sd0 = 1 / np.sqrt(1 - 0.9 * 0.9)
    res = orc.pf_ar1(2000, y, 0.9, 1.0, 0.5, sd0, (11, 0), (12, 0), scheme)
    assert res["loglik"] == GOLD[f"pf_{scheme}_loglik"][0]
    assert np.array_equal(res["resampled"], GOLD[f"pf_{scheme}_resampled"])
    assert np.array_equal(res["anc"][res["resampled"] == 1].astype(np.uint16), GOLD[f"pf_{scheme}_anc"])
    assert same_bits(res["x"], GOLD[f"pf_{scheme}_x"])
    assert np.array_equal(res["ess"], GOLD[f"pf_{scheme}_ess"])


def test_rep_index_invariants(orc):
    """Structural invariants the reference's own example checks
    (example/algorithm/include/algorithm_resample_transform.hpp:37-80)."""
    rng = np.random.default_rng(5)
    for N, M in ((1000, 1000), (1000, 600), (600, 1000), (1, 5), (5, 1)):
        W = rng.random(N)
        W /= W.sum()
        rep = orc.resample(2, O.Engine.make(1, key=(3,)), W, M)
        assert int(rep.sum()) == M
        idx = orc.rep_index(rep, M)
        K = min(N, M)
        for i in range(K):
            if rep[i] > 0:
                assert idx[i] == i
        counts = np.bincount(idx.astype(np.int64), minlength=N)
        assert np.array_equal(counts, rep.astype(np.int64))


def test_kalman_gradient_matches_finite_differences(orc):
    y = GOLD["pf_y"]
    ll, g = orc.kalman_ar1(y, 0.9, 1.0, 0.5)
    h = 1e-6
    for k in range(3):
        p = [0.9, 1.0, 0.5]
        p[k] += h
        lp, _ = orc.kalman_ar1(y, *p)
        p[k] -= 2 * h
        lm, _ = orc.kalman_ar1(y, *p)
        assert abs((lp - lm) / (2 * h) - g[k]) < 1e-5 * max(1.0, abs(g[k]))


@pytest.mark.skipif(not os.path.isdir(os.path.join(O.REF_ROOT, "example", "random")),
                    reason="reference source tree not present")
@pytest.mark.parametrize("kind,name", [(1, "philox4x32"), (2, "philox4x32_64"), (3, "threefry4x64"),
                                       (4, "threefry4x64_64"), (5, "ars"), (6, "ars_64")])
def test_known_answer_files(orc, kind, name):
    kat = np.loadtxt(os.path.join(O.REF_ROOT, "example", "random", f"random_{name}.data"), dtype=np.uint64)
    w = orc.rand(O.Engine.make(kind, key=(1,)), 1000)
    assert np.array_equal(w.astype(np.uint64), kat)


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built")
def test_oracle_vs_compiled_reference_randomized(orc):
    ref_aesni = O.CPUPath("ref")
    ref_generic = O.CPUPath("ref_generic")
    rng = np.random.default_rng(11)
    for _ in range(40):
        kind = int(rng.integers(1, 7))
        M = O.WORDS_PER_BLOCK[kind]
        idx = int(rng.integers(0, M + 1))
        ctr = (int(rng.integers(0, 2**63)),)
        n = int(rng.integers(0, 3000))
        a = O.Engine.make(kind, key=(int(rng.integers(0, 2**32)), 3), ctr=ctr, index=idx)
        b = a.copy()
        ref = ref_generic if kind in (5, 6) else ref_aesni
        assert same_bits(orc.rand(a, n), ref.rand(b, n))
        assert a.state() == b.state()
        if kind in (1, 3, 5):
            f64 = bool(rng.integers(0, 2))
            a2, b2 = a.copy(), b.copy()
            n2 = int(rng.integers(1, 5000))
            assert same_bits(orc.normal(a2, f64, n2, 0.5, 1.5), ref.normal(b2, f64, n2, 0.5, 1.5))
            assert a2.state() == b2.state()
            alpha = float(rng.uniform(0.1, 12))
            assert same_bits(orc.gamma(a, f64, n2, alpha, 0.7), ref.gamma(b, f64, n2, alpha, 0.7))
            assert a.state() == b.state()


def test_kalman_gradient_vs_finite_differences(orc):
    """The Kalman oracle's forward-mode gradient against central differences."""
    e = O.Engine.make(1, key=(7,))
    for (phi, sx, sy) in ((0.9, 1.0, 0.5), (0.55, 1.7, 0.25), (0.97, 0.6, 0.9)):
        y = np.concatenate([[0.0], np.cumsum(orc.normal(e, True, 200, 0.0, 1.0)) * 0.1])
        _, g = orc.kalman_ar1(y, phi, sx, sy)
        h = 1e-6
        for k in range(3):
            p = [phi, sx, sy]
            p[k] += h
            lp, _ = orc.kalman_ar1(y, *p)
            p[k] -= 2 * h
            lm, _ = orc.kalman_ar1(y, *p)
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_weighted_estimate_oracle_pin():
    """The oracle's dgemv-order estimate against the exactly rounded sum
    (math.fsum), within the FP64 error bound of an n-term sum, both layouts
    identical; and against the installed BLAS's dgemv (any order) within the
    same bound."""
    import math

    from scipy.linalg import blas

    orc = O.CPUPath("oracle")
    rng = np.random.default_rng(5)
    for n, d in ((1, 1), (1000, 3), (5000, 17)):
        W = rng.random(n)
        W /= W.sum()
        u = rng.normal(size=(n, d)) * 2 - 1
        got = orc.weighted_estimate(u, W)
        assert np.array_equal(got, orc.weighted_estimate(np.ascontiguousarray(u.T), W, col_major=True))
        lib = blas.dgemv(1.0, u, W, trans=1)
        for j in range(d):
            bound = n * 2.0**-53 * float(np.sum(np.abs(W * u[:, j])))
            assert abs(got[j] - math.fsum(W * u[:, j])) <= bound
            assert abs(got[j] - lib[j]) <= 2 * bound


def test_library_kalman_matches_oracle():
    """The package's vectorised Kalman filter (the yardstick the bench
    reports against) equals the oracle's scalar one."""
    from mckl_b200.kalman import kalman_ar1

    orc = O.CPUPath("oracle")
    rng = np.random.default_rng(8)
    F, T = 5, 200
    y = rng.normal(size=(F, T + 1))
    phi = rng.uniform(0.5, 0.99, F)
    sx = rng.uniform(0.5, 2, F)
    sy = rng.uniform(0.2, 1, F)
    ll, g = kalman_ar1(y, phi, sx, sy)
    for f in range(F):
        l1, g1 = orc.kalman_ar1(y[f], phi[f], sx[f], sy[f])
        assert abs(ll[f] - l1) <= 1e-10 * abs(l1)
        assert np.allclose(g[f], g1, rtol=1e-9, atol=1e-9)
