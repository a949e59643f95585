"""GPU parity at the RNG + distributions configuration, at full size.

Threefry4x64-20 and ARS-5 seeded 42, 2^28 values per call, as the benchmark
draws them: raw u32 words, canonical U01 in float and double, Normal(0, 1) and
Exponential(1) in float and double, and Gamma(alpha_b, 1) over 65 536 blocks
of 4096 samples with alpha_b ~ U[0.5, 10] per block (block b an independent
stream at counter (0, b)).

Words and U01 values must be bit-identical; Normal and Exponential within
2 ULP (double) or 1e-6 relative (float); Gamma under the bars of
test_gpu_gamma (double: >= 99 % bit-identical and every value within 1e-12
relative; float: >= 90 % bit-identical, >= 99 % within 1e-6 and every value
within 2e-5 relative).  A full CPU recomputation of the 2^28-value streams is
too slow for a test, so the oracle checks the first and last windows and 32
random windows of every call (the oracle engine positioned at the window's
first word, exactly as the reference's rng.ctr() positioning does), and the
engine state after each call.  Gamma is checked block for block, all 65 536
blocks (the oracle runs its blocks on every host thread).
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402

N = 1 << 28
KINDS = {3: "Threefry4x64", 5: "ARS"}
GAMMA_BLOCK = 4096


@pytest.fixture(scope="module")
def env():
    require_cuda()
    import mckl_b200 as mb

    O.build()
    return mb, O.CPUPath("oracle")


def engine_at(orc, kind, word):
    """An oracle engine seeded 42 whose next word is word `word` of the stream."""
    M = O.WORDS_PER_BLOCK[kind]
    e = O.Engine.make(kind, key=(42,), ctr=(word // M,))
    if word % M:
        orc.rand(e, word % M)
    return e


def windows(n, width, align, seed):
    rng = np.random.default_rng(seed)
    pos = [int(p) // align * align for p in rng.integers(0, n - width, 32)]
    return [0, n - width] + pos


def state_after(orc, kind, words):
    """The reference engine's state after a batch call that consumed `words`
    words from a fresh seed (a batch call ends with the next block buffered),
    from the oracle positioned one block before the end."""
    M = O.WORDS_PER_BLOCK[kind]
    assert words % M == 0
    e = engine_at(orc, kind, words - M)
    orc.rand(e, M)
    return e.state()


def ulps(a, b):
    d = np.abs(a - b)
    return np.where(d == 0, 0.0, d / np.spacing(np.maximum(np.abs(a), np.abs(b))))


@pytest.mark.parametrize("kind", [3, 5])
def test_c2_streams_and_transforms(env, kind):
    mb, orc = env
    buf32 = torch.empty(N, dtype=torch.int32, device="cuda")
    buf64 = torch.empty(N, dtype=torch.float64, device="cuda")
    f32 = buf32.view(torch.float32)
    fresh = lambda: mb.ENGINES[KINDS[kind]](42)  # noqa: E731

    # raw words
    g = fresh()
    mb.rand(g, N, buf32)
    assert g.state_tuple() == state_after(orc, kind, N)
    for p in windows(N, 1024, 1, 1):
        got = buf32[p:p + 1024].cpu().numpy().view(np.uint32)
        assert np.array_equal(got, orc.rand(engine_at(orc, kind, p), 1024)), ("raw", p)

    # canonical U01: one word per float, two per double
    for f64, buf, wpv in ((False, f32, 1), (True, buf64, 2)):
        g = fresh()
        mb.u01_canonical_distribution(g, N, buf)
        assert g.state_tuple() == state_after(orc, kind, N * wpv)
        for p in windows(N, 1024, 1, 2):
            got = buf[p:p + 1024].cpu().numpy()
            want = orc.u01(engine_at(orc, kind, p * wpv), "canonical", f64, 1024)
            assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), ("u01", f64, p)

    # Normal(0, 1): chunks of 1024 (double) / 2048 (float) values, one word each
    for f64, buf, K in ((False, f32, 2048), (True, buf64, 1024)):
        g = fresh()
        mb.normal_distribution(g, N, buf)
        assert g.state_tuple() == state_after(orc, kind, N)
        worst = 0.0
        for p in windows(N, K, K, 3):
            got = buf[p:p + K].cpu().numpy()
            want = orc.normal(engine_at(orc, kind, p), f64, K)
            if f64:
                worst = max(worst, float(ulps(got, want).max()))
            else:
                rel = np.abs(got.astype(np.float64) - want) / np.abs(want.astype(np.float64))
                worst = max(worst, float(rel.max()))
        assert worst <= (2 if f64 else 1e-6), ("normal", f64, worst)

    # Exponential(1): one word per value
    for f64, buf in ((False, f32), (True, buf64)):
        g = fresh()
        mb.exponential_distribution(g, N, buf)
        assert g.state_tuple() == state_after(orc, kind, N)
        for p in windows(N, 1024, 1, 4):
            got = buf[p:p + 1024].cpu().numpy()
            want = orc.exponential(engine_at(orc, kind, p), f64, 1024)
            if f64:
                assert ulps(got, want).max() <= 2, ("exponential", p)
            else:
                rel = np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want.astype(np.float64)), 1e-30)
                assert rel.max() <= 1e-6, ("exponential f32", p)
    del buf32, buf64
    torch.cuda.empty_cache()


def gamma_shapes(orc, nblocks):
    """alpha_b ~ U[0.5, 10]: canonical uniforms of Philox4x32(43)."""
    u = orc.u01(O.Engine.make(O.PHILOX4X32, key=(43,)), "canonical", True, nblocks)
    return 0.5 + 9.5 * u


@pytest.mark.parametrize("kind", [3, 5])
def test_c2_gamma_all_blocks(env, kind):
    mb, orc = env
    nb = N // GAMMA_BLOCK
    alpha = gamma_shapes(orc, nb)
    threads = os.cpu_count() or 1
    for f64 in (False, True):
        dt = "f64" if f64 else "f32"
        g = mb.ENGINES[KINDS[kind]](42)
        before = g.state_tuple()
        got_dev = mb.gamma_blocks(g, GAMMA_BLOCK, alpha, dtype=dt)
        assert g.state_tuple() == before  # the per-block streams do not advance the caller's engine
        exact = 0
        within = 0
        worst = 0.0
        step = 8192  # blocks per oracle batch (bounded host memory)
        for b0 in range(0, nb, step):
            b1 = min(nb, b0 + step)
            # block b is its own stream: the engine at counter (0, b), nothing buffered
            want = orc.gamma_blocks_from(O.Engine.make(kind, key=(42,)), f64, b0, GAMMA_BLOCK, alpha[b0:b1], 1.0,
                                         nthreads=threads)
            got = got_dev[b0 * GAMMA_BLOCK:b1 * GAMMA_BLOCK].cpu().numpy()
            bits = np.uint64 if f64 else np.uint32
            exact += int(np.sum(got.view(bits) == want.view(bits)))
            rel = np.abs(got.astype(np.float64) - want.astype(np.float64)) / np.maximum(
                np.abs(want.astype(np.float64)), 1e-300)
            within += int(np.sum(rel <= 1e-6))
            worst = max(worst, float(rel.max()))
        frac_exact = exact / N
        if f64:
            assert frac_exact >= 0.99 and worst <= 1e-12, (kind, dt, frac_exact, worst)
        else:
            assert frac_exact >= 0.90 and worst <= 2e-5 and within / N >= 0.99, (kind, dt, frac_exact, worst)
        del got_dev
        torch.cuda.empty_cache()

