"""GPU parity for Gamma(alpha, beta) (random/gamma_distribution.hpp:57-302)
through the C ABI, against the CPU oracle (pinned to the reference's own
outputs in test_oracle_pins) and the golden fixtures made by the compiled
reference.

What must agree exactly: the engine state after every call, and the
acceptance pattern -- every value sits at the same position as in the
reference's stream, so a single flipped accept/reject decision (which would
shift the rest of the stream) fails the test.  Values: the device and glibc
log/exp/sin/cos differ in the last place for a small fraction of arguments
(the device's are correctly rounded), and Gamma's transforms amplify such a
difference: x = exp(c log u) carries |c log u| times the relative error of
the log.  So the bars are: fp64 -- at least 99 % of values bit-identical and
every value within 1e-12 relative; fp32 -- at least 90 % bit-identical and
every value within 2e-5 relative (1e-6 relative for at least 99 %).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402

GOLD = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "golden.npz"))
KINDS = {1: "Philox4x32", 2: "Philox4x32_64", 3: "Threefry4x64", 4: "Threefry4x64_64", 5: "ARS", 6: "ARS_64"}


@pytest.fixture(scope="module")
def env():
    require_cuda()
    import mckl_b200 as mb

    O.build()
    return mb, O.CPUPath("oracle")


def pair(mb, kind, key=(42,), ctr=(0,), index=None):
    e = O.Engine.make(kind, key=key, ctr=ctr, index=index)
    g = mb.ENGINES[KINDS[kind]]()
    g.load_state(list(e.ctr), list(e.key), list(e.tweak), e.index)
    return g, e


def check_values(got, want, f64, what):
    assert got.shape == want.shape
    same = got.view(np.uint8).reshape(len(got), -1) == want.view(np.uint8).reshape(len(want), -1)
    exact = float(np.mean(np.all(same, axis=1))) if len(got) else 1.0
    a = got.astype(np.float64)
    b = want.astype(np.float64)
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    if f64:
        assert exact >= 0.99 and rel.max(initial=0) <= 1e-12, (what, exact, rel.max(initial=0))
    else:
        assert exact >= 0.90 and rel.max(initial=0) <= 2e-5, (what, exact, rel.max(initial=0))
        assert np.mean(rel <= 1e-6) >= 0.99, what
    return exact, float(rel.max(initial=0))


@pytest.mark.parametrize("kind", range(1, 7))
def test_gamma_vs_oracle(env, kind):
    mb, orc = env
    for f64 in (False, True):
        dt = "f64" if f64 else "f32"
        for alpha in (0.3, 0.55, 0.7, 1.0, 2.5, 9.7):
            for (n, idx) in ((4096, None), (1, 2), (2049, 1), (5000, None)):
                g, e = pair(mb, kind, index=idx)
                want = orc.gamma(e, f64, n, alpha, 1.5)
                got = mb.gamma_distribution(g, n, alpha=alpha, beta=1.5, dtype=dt).cpu().numpy()
                check_values(got, want, f64, (kind, dt, alpha, n, idx))
                assert g.state_tuple() == e.state(), (kind, dt, alpha, n, idx)


@pytest.mark.parametrize("kind", [1, 3, 5])
def test_gamma_golden(env, kind):
    mb, orc = env
    for f64 in (False, True):
        for alpha in (0.3, 0.7, 1.0, 2.5, 9.7):
            g, e = pair(mb, kind, key=(42,))
            got = mb.gamma_distribution(g, 4096, alpha=alpha, beta=1.0, dtype="f64" if f64 else "f32").cpu().numpy()
            check_values(got, GOLD[f"gamma_{kind}_{int(f64)}_{alpha}"], f64, (kind, f64, alpha))
            orc.gamma(e, f64, 4096, alpha, 1.0)  # its state is pinned to the fixture's
            assert g.state_tuple() == e.state()


def test_gamma_consecutive_calls(env):
    """Two calls in a row continue the stream exactly as the reference does."""
    mb, orc = env
    g, e = pair(mb, 1, key=(7,))
    for (n, alpha) in ((3000, 2.5), (777, 0.4), (4096, 0.8), (10, 1.0)):
        want = orc.gamma(e, True, n, alpha, 1.0)
        got = mb.gamma_distribution(g, n, alpha=alpha, dtype="f64").cpu().numpy()
        check_values(got, want, True, (n, alpha))
        assert g.state_tuple() == e.state()


@pytest.mark.parametrize("kind", [3, 5])
def test_gamma_blocks(env, kind):
    """The per-block form: 128 blocks of 4096 with alpha ~ U[0.5, 10]."""
    mb, orc = env
    rng = np.random.default_rng(11)
    alpha = 0.5 + 9.5 * rng.random(128)
    for f64 in (False, True):
        g, e = pair(mb, kind, key=(42,))
        want = orc.gamma_blocks(e, f64, 4096, alpha, 1.0)
        got = mb.gamma_blocks(g, 4096, alpha, dtype="f64" if f64 else "f32").cpu().numpy()
        check_values(got, want, f64, (kind, f64))
        assert g.state_tuple() == e.state()  # the caller's engine is not advanced
