"""CPU-side checks of the C ABI boundary: the shared library loads, exports
every entry point declared in include/*.h, and its host-only engine state
operations follow the reference's CounterEngine arithmetic."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(mckl_b200_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import mckl_b200 as mb

    lib = mb.raw_lib()
    names = declared_symbols()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_in_tree():
    import mckl_b200 as mb

    assert os.path.dirname(mb.lib_path()) == os.path.join(ROOT, "mckl_b200")


@pytest.mark.parametrize("kind", range(1, 7))
def test_seed_and_discard_follow_the_stream(kind):
    import mckl_b200 as mb

    orc = O.CPUPath("oracle")
    cls = {1: mb.Philox4x32, 2: mb.Philox4x32_64, 3: mb.Threefry4x64, 4: mb.Threefry4x64_64,
           5: mb.ARS, 6: mb.ARS_64}[kind]
    M = O.WORDS_PER_BLOCK[kind]
    for k in (0, 1, M - 1, M, M + 1, 5 * M + 3, 1000):
        g = cls(42)
        e = O.Engine.make(kind, key=(42,))
        assert g.state_tuple() == e.state()
        g.discard(k)
        # after discard(k), the stream continues at word k
        tail = orc.rand(O.Engine.make(kind, key=(42,)), k + 8)[k:]
        e2 = O.Engine.make(kind)
        e2.ctr[0], e2.key[0], e2.index = g.state.ctr[0], 42, g.state.index
        assert np.array_equal(orc.rand(e2, 8), tail)


def test_bad_arguments_are_rejected_without_gpu_work():
    import mckl_b200 as mb

    lib = mb.raw_lib()
    st = mb.EngineState()
    assert lib.mckl_b200_engine_seed(ctypes.byref(st), 99, 1) == -1
    assert b"kind" in lib.mckl_b200_last_error()
