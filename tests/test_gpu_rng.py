"""GPU parity: raw engine streams, U01, Normal and Exponential through the C ABI
against the CPU oracle (itself pinned to the reference in test_oracle_pins).

Integer words and the U01 conversions (exact products, one rounding) must be
bit-identical, engine state included.  Normal / Exponential go through device
log / sqrt / sin / cos, so values are compared with the configuration's
tolerances:
  fp64: at most 2 ULP, fp32: relative error at most 1e-6, both measured
  against max(|value|, |mean|) -- a value mean + sd z close to zero is a
  cancellation, and there the error is set by the size of the two terms, not
  of their difference (for mean = 0 this is the plain per-value bound).
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


KINDS = {1: "Philox4x32", 2: "Philox4x32_64", 3: "Threefry4x64", 4: "Threefry4x64_64", 5: "ARS", 6: "ARS_64"}


def pair(mb, kind, key=(42,), ctr=(0,), index=None):
    e = O.Engine.make(kind, key=key, ctr=ctr, index=index)
    g = mb.ENGINES[KINDS[kind]]()
    g.load_state(list(e.ctr), list(e.key), list(e.tweak), e.index)
    return g, e


def same_state(g, e):
    return g.state_tuple() == e.state()


def ulps(a, b):
    a = a.astype(np.float64) if a.dtype == np.float32 else a
    b = b.astype(np.float64) if b.dtype == np.float32 else b
    return np.abs(a - b) / np.spacing(np.maximum(np.abs(a), np.abs(b)))


@pytest.mark.parametrize("kind", range(1, 7))
def test_rand_streams(env, kind):
    mb, orc = env
    M = O.WORDS_PER_BLOCK[kind]
    # low counter words that do and do not carry into bit 32 within a call
    # (the Philox fill folds the block-independent rounds only when they do
    # not), and nonzero upper words
    for (ctr, idx) in (((0,), None), ((5,), 0), ((7,), 1), ((9,), M - 1), ((2**64 - 2, 3), None), ((2**64 - 1,), 1),
                       ((2**32 - 3,), None), ((2**33 + 7, 12345), None), ((2**40 + 3, 2**50 + 9), 2)):
        for n in (0, 1, 3, 5, 17, 1000, 4096 * 3 + 5, 1 << 20):
            g, e = pair(mb, kind, key=(42, 5, 3, 1), ctr=ctr, index=idx)
            want = orc.rand(e, n)
            got = mb.words_to_numpy(mb.rand(g, n), g.result_bits())
            assert np.array_equal(got, want), (ctr, idx, n)
            assert same_state(g, e), (ctr, idx, n)


@pytest.mark.parametrize("kind", range(1, 7))
def test_rand_misaligned_output(env, kind):
    mb, orc = env
    g, e = pair(mb, kind, key=(42,))
    n = 10001
    buf = mb.empty_words(g, n + 3)
    mb.rand(g, n, buf[1:])
    torch.cuda.synchronize()
    got = mb.words_to_numpy(buf, g.result_bits())[1:n + 1]
    assert np.array_equal(got, orc.rand(e, n))


def test_generator_level_kernels(env):
    mb, orc = env
    n = 12345
    r = torch.empty(n * 4, dtype=torch.int32, device="cuda")
    c = mb.philox4x32_kernel((7, 0), n, r, (42, 0))
    e = O.Engine.make(1, key=(42,), ctr=(7,))
    assert np.array_equal(mb.words_to_numpy(r, 32), orc.rand(e, n * 4))
    assert c == (7 + n, 0)
    r = torch.empty(n * 8, dtype=torch.int32, device="cuda")
    c = mb.threefry4x64_kernel((2**64 - 5, 0, 0, 0), n, r, (42, 1, 2, 3), tweak=(0, 0))
    e = O.Engine.make(3, key=(42, 1, 2, 3), ctr=(2**64 - 5,))
    assert np.array_equal(mb.words_to_numpy(r, 32), orc.rand(e, n * 8))
    assert c == ((2**64 - 5 + n) % 2**64, 1, 0, 0)
    r = torch.empty(n * 4, dtype=torch.int32, device="cuda")
    mb.ars_kernel((0, 0), n, r, (42, 9, 8, 7))
    e = O.Engine.make(5, key=(42, 9, 8, 7))
    assert np.array_equal(mb.words_to_numpy(r, 32), orc.rand(e, n * 4))


@pytest.mark.parametrize("kind", range(1, 7))
def test_u01_bit_exact(env, kind):
    mb, orc = env
    fns = {"canonical": mb.u01_canonical_distribution, "cc": mb.u01_cc_distribution,
           "co": mb.u01_co_distribution, "oc": mb.u01_oc_distribution, "oo": mb.u01_oo_distribution}
    for var, fn in fns.items():
        for dt in ("f32", "f64"):
            for (ctr, idx, n) in (((3,), None, 5000), ((3,), 1, 4099), ((3,), 2, 1 << 18), ((2**32 - 700,), None, 5000),
                                  ((2**35 + 1, 7), None, 4096 * 4 + 12)):
                g, e = pair(mb, kind, ctr=ctr, index=idx)
                want = orc.u01(e, var, dt == "f64", n)
                got = fn(g, n, dtype=dt).cpu().numpy()
                assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), (var, dt, ctr, idx, n)
                assert same_state(g, e), (var, dt, ctr, idx, n)


@pytest.mark.parametrize("kind", range(1, 7))
def test_normal(env, kind):
    mb, orc = env
    worst = {}
    for dt in ("f32", "f64"):
        for (idx, n, mean, sd) in ((None, 1 << 16, 0.0, 1.0), (1, 4097, 1.5, 2.0), (None, 2049, 0.0, 3.0),
                                   (2, 7, -1.0, 0.5), (None, 1, 0.0, 1.0)):
            g, e = pair(mb, kind, index=idx)
            want = orc.normal(e, dt == "f64", n, mean, sd)
            got = mb.normal_distribution(g, n, mean=mean, stddev=sd, dtype=dt).cpu().numpy()
            assert same_state(g, e)
            if dt == "f64":
                # ULPs of max(|value|, |mean|): see the module docstring
                scale = np.maximum(np.abs(want), abs(mean))
                u = np.abs(got - want) / np.spacing(scale)
                worst[(dt, n)] = float(u.max())
                assert u.max() <= 2, (n, mean, sd, u.max())
            else:
                scale = np.maximum(np.abs(want.astype(np.float64)), max(abs(mean), 1e-30))
                rel = np.abs(got.astype(np.float64) - want) / scale
                worst[(dt, n)] = float(rel.max())
                assert rel.max() <= 1e-6, (n, rel.max())


@pytest.mark.parametrize("kind", range(1, 7))
def test_exponential(env, kind):
    mb, orc = env
    for dt in ("f32", "f64"):
        for (idx, n, lam) in ((None, 1 << 16, 1.0), (3, 5001, 2.5)):
            g, e = pair(mb, kind, index=idx)
            want = orc.exponential(e, dt == "f64", n, lam)
            got = mb.exponential_distribution(g, n, lam=lam, dtype=dt).cpu().numpy()
            assert same_state(g, e)
            if dt == "f64":
                assert ulps(got, want).max() <= 2
            else:
                rel = np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want.astype(np.float64)), 1e-30)
                assert rel.max() <= 1e-6


def test_full_size_philox_c1(env):
    """Config C1 at full size: Philox4x32(42), 2^26 words then 2^24 U01OO doubles
    from the same stream.  The oracle checks a prefix, a suffix and random
    positions of each (a full CPU recomputation is too slow for a test), and
    the engine state after both calls must match the reference's arithmetic."""
    mb, orc = env
    g, e = pair(mb, 1, key=(42,))
    words = mb.words_to_numpy(mb.rand(g, 1 << 26), 32)
    u = mb.u01_oo_distribution(g, 1 << 24, dtype="f64").cpu().numpy()
    assert np.array_equal(words[:4], np.array([4242219303, 1404726525, 2207210094, 1951270651], dtype=np.uint32))
    rng = np.random.default_rng(0)
    for pos in list(rng.integers(0, (1 << 26) - 64, 32)) + [0, (1 << 26) - 64]:
        blk = pos // 4
        ep = O.Engine.make(1, key=(42,), ctr=(blk,))
        want = orc.rand(ep, 64 + pos % 4)[pos % 4:]
        assert np.array_equal(words[pos:pos + 64], want)
    ep = O.Engine.make(1, key=(42,), ctr=((1 << 24),))
    assert np.array_equal(u[:1000].view(np.uint64), orc.u01(ep, "oo", True, 1000).view(np.uint64))
    fresh = mb.u01_oo_distribution(mb.Philox4x32(42), 1, dtype="f64").cpu().numpy()
    assert fresh[0] == 0.98771865095477551
    # state: 2^26 words -> ctr 2^24 + 1 buffered, index 0; then 2^24 more words
    orc.rand(e, 1 << 26)
    orc.u01(e, "oo", True, 1 << 24)
    assert same_state(g, e)
