"""Engine states in the reference's text form (CounterEngine operator<< /
operator>>, random/counter.hpp:235-272), host-only entry points
mckl_b200_engine_save / _load, against the compiled reference: the text the
library writes equals the reference's token for token (the buffered results
only where the buffer is in use), the reference reads it back into the same
state, and the library reads the reference's text into the same state."""
import ctypes

import numpy as np
import pytest

import oracle as O


@pytest.fixture(scope="module")
def env():
    if not O.have_ref():
        pytest.skip("reference build missing")
    import mckl_b200 as mb

    O.build(ref=True)
    lib = mb.raw_lib()
    lib.mckl_b200_engine_save.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_size_t)]
    lib.mckl_b200_engine_load.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_char_p]
    return lib, O.CPUPath("ref_generic")


def save(lib, e):
    n = ctypes.c_size_t()
    assert lib.mckl_b200_engine_save(ctypes.byref(e), None, 0, ctypes.byref(n)) == 0
    buf = ctypes.create_string_buffer(n.value + 1)
    assert lib.mckl_b200_engine_save(ctypes.byref(e), buf, n.value + 1, ctypes.byref(n)) == 0
    return buf.value.decode()


def states(kind, rng):
    M = O.WORDS_PER_BLOCK[kind]
    for _ in range(12):
        key = tuple(int(v) for v in rng.integers(0, 2**32, 4)) if kind in (5, 6) else \
            (tuple(int(v) for v in rng.integers(0, 2**63, 4)) if kind in (3, 4) else
             tuple(int(v) for v in rng.integers(0, 2**32, 2)))
        ctr = tuple(int(v) for v in rng.integers(0, 2**63, 2))
        idx = int(rng.integers(0, M + 1))
        tweak = tuple(int(v) for v in rng.integers(0, 2**63, 2)) if kind in (3, 4) else (0, 0)
        yield O.Engine.make(kind, key=key, ctr=ctr, index=idx, tweak=tweak)


@pytest.mark.parametrize("kind", range(1, 7))
def test_save_matches_reference_text(env, kind):
    lib, ref = env
    M = O.WORDS_PER_BLOCK[kind]
    for e in states(kind, np.random.default_rng(kind)):
        ours = save(lib, e).split()
        theirs = ref.engine_text(e).split()
        assert len(ours) == len(theirs)
        if e.index < M:
            assert ours == theirs, (ours, theirs)
        else:
            assert ours[0] == theirs[0] and ours[M + 1:] == theirs[M + 1:], (ours, theirs)
        # the reference reads our text and writes it back unchanged
        assert ref.engine_text_roundtrip(kind, " ".join(ours)).split() == ours


@pytest.mark.parametrize("kind", range(1, 7))
def test_load_reference_text(env, kind):
    lib, ref = env
    for e in states(kind, np.random.default_rng(100 + kind)):
        text = ref.engine_text(e)
        got = O.Engine.make(kind)
        if e.index < O.WORDS_PER_BLOCK[kind]:
            assert lib.mckl_b200_engine_load(ctypes.byref(got), kind, text.encode()) == 0
            assert got.state() == e.state()


def test_load_rejects_foreign_buffer(env):
    lib, ref = env
    e = O.Engine.make(1, key=(5, 6), ctr=(9, 0), index=1)
    tok = save(lib, e).split()
    tok[1] = str((int(tok[1]) + 1) % 2**32)  # a buffered result the counter does not produce
    got = O.Engine.make(1)
    assert lib.mckl_b200_engine_load(ctypes.byref(got), 1, " ".join(tok).encode()) != 0
    assert lib.mckl_b200_engine_load(ctypes.byref(got), 1, b"not an engine") != 0


def test_load_unused_buffer_any_words(env):
    """index == M: the buffer is not in use, whatever words the text holds."""
    lib, ref = env
    for kind in range(1, 7):
        M = O.WORDS_PER_BLOCK[kind]
        e = O.Engine.make(kind, ctr=(3, 4), index=M)
        tok = save(lib, e).split()
        tok[1:M + 1] = [str(7 * i + 1) for i in range(M)]
        got = O.Engine.make(kind)
        assert lib.mckl_b200_engine_load(ctypes.byref(got), kind, " ".join(tok).encode()) == 0
        assert got.state()[:2] == e.state()[:2] and got.index == M


def test_python_engine_text_after_draws(env):
    """str(rng) / from_text on engines advanced by host-side bookkeeping
    (discard), for every kind: equal to the reference's text after the same
    discards, and read back into the same state."""
    import mckl_b200 as mb

    lib, ref = env
    classes = {1: mb.Philox4x32, 2: mb.Philox4x32_64, 3: mb.Threefry4x64, 4: mb.Threefry4x64_64,
               5: mb.ARS, 6: mb.ARS_64}
    for kind, cls in classes.items():
        for skip in (0, 1, 3, 7, 1000003):
            g = cls(2024)
            g.discard(skip)
            text = str(g)
            st = g.state_tuple()
            e = O.Engine.make(kind, key=st[1], ctr=st[0][:2] if kind not in (3, 4) else st[0],
                              index=st[3], tweak=st[2])
            if g.index < O.WORDS_PER_BLOCK[kind]:
                assert text.split() == ref.engine_text(e).split()
            back = cls.from_text(text)
            assert back.state_tuple() == st
            with pytest.raises(mb.MCKLB200Error):
                cls.from_text(text.replace(text.split()[0], "99", 1))
