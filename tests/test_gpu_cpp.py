"""The C++ host interface (include/mckl_b200.hpp) on the GPU.

1. The reference's own mckl::CounterEngine and distributions driven by the
   B200 generators equal the reference's engines (oracle/_ref/
   shim_reference_test, built by `make -C oracle shim` where the reference
   headers are present).
2. The device-side C++ API, compiled here from tests/cpp/shim_device_test.cpp,
   agrees with the oracle.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def gpu():
    require_cuda()


def test_reference_counter_engine_over_b200_generators(gpu):
    exe = os.path.join(ROOT, "oracle", "_ref", "shim_reference_test")
    if not os.path.exists(exe):
        pytest.skip("shim_reference_test not built (needs the reference headers)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("equal") == 3


def test_device_cpp_api(gpu):
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "shim_device_test")
        cmd = ["g++", "-O2", "-std=c++14", f"-I{ROOT}/include", f"-I{CUDA}/include",
               os.path.join(ROOT, "tests", "cpp", "shim_device_test.cpp"), "-o", exe,
               f"-L{ROOT}/mckl_b200", "-lmckl_b200", f"-Wl,-rpath,{ROOT}/mckl_b200", f"-L{CUDA}/lib64", "-lcudart",
               f"-Wl,-rpath,{CUDA}/lib64"]
        subprocess.run(cmd, check=True, capture_output=True)
        out = os.path.join(d, "out.bin")
        r = subprocess.run([exe, out], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        raw = open(out, "rb").read()
    N = 3000
    words = np.frombuffer(raw, dtype=np.uint32, count=10000, offset=0)
    z = np.frombuffer(raw, dtype=np.float64, count=4097, offset=40000)
    W = np.frombuffer(raw, dtype=np.float64, count=N, offset=40000 + 4097 * 8)
    idx = np.frombuffer(raw, dtype=np.uint64, count=N, offset=40000 + 4097 * 8 + N * 8)
    ess = np.frombuffer(raw, dtype=np.float64, count=1, offset=40000 + 4097 * 8 + 2 * N * 8)[0]
    orc = O.CPUPath("oracle")
    e = O.Engine.make(1, key=(42,))
    assert np.array_equal(words, orc.rand(e, 10000))
    zr = orc.normal(e, True, 4097)
    assert np.max(np.abs(z - zr) / np.spacing(np.abs(zr))) <= 2
    v = np.array([((i * 7919) % 1000) / 100.0 - 5.0 for i in range(N)])
    Wr, essr = orc.weight_set_log(v)
    assert np.max(np.abs(W - Wr) / np.spacing(Wr)) <= 2
    assert abs(ess - essr) <= 1e-13 * essr
    rep = orc.resample(2, O.Engine.make(1, key=(9,)), Wr)
    assert np.array_equal(idx, orc.rep_index(rep))
