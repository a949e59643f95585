"""The model hook of the batched filters (include/mckl_b200_batched.cuh): a
user's model struct instantiates the persistent kernel in the user's own
translation unit.  tests/cpp/batched_model_test.cu writes the AR(1) model as
a user would (its own struct, the explicit roundings of Math<R>) and runs it
through mckl_b200::batched_run_model in FP32 and FP64; its log-likelihoods
and resampling counts must equal the library's built-in AR(1) filters'
(mckl_b200_batched_run) bit for bit, on filters of uneven sizes."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_user_model_equals_builtin_ar1():
    require_cuda()
    import mckl_b200 as mb

    w = mb.batched_workload(F=24, T=60, seed=17, nmin=300, nmax=6000)
    F, T = len(w["N"]), w["y"].shape[1] - 1
    threshold = 0.5
    want = {}
    for fp64 in (False, True):
        b = mb.BatchedFilters(w["N"], w["y"], w["phi"], w["sx"], w["sy"], w["mkeys"], w["rkeys"],
                              threshold=threshold, fp64=fp64)
        b.config(256, 4)
        b.run()
        want[fp64] = b.results()
        b.close()
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "batched_model_test")
        r = subprocess.run([os.path.join(CUDA, "bin", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                            "-std=c++17", "--expt-relaxed-constexpr", f"-I{ROOT}/include",
                            f"-I{ROOT}/mckl_b200/csrc", os.path.join(ROOT, "tests", "cpp", "batched_model_test.cu"),
                            "-o", exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
        inp, out = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(inp, "wb") as f:
            f.write(np.array([F, T], dtype=np.int32).tobytes())
            f.write(np.array([threshold], dtype=np.float64).tobytes())
            f.write(np.ascontiguousarray(w["N"], dtype=np.uint64).tobytes())
            for k in ("phi", "sx", "sy"):
                f.write(np.ascontiguousarray(w[k], dtype=np.float64).tobytes())
            f.write(np.ascontiguousarray(w["mkeys"], dtype=np.uint32).tobytes())
            f.write(np.ascontiguousarray(w["rkeys"], dtype=np.uint32).tobytes())
            f.write(np.ascontiguousarray(w["y"], dtype=np.float64).tobytes())
        r = subprocess.run([exe, inp, out], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        raw = open(out, "rb").read()
    o = 0
    got = {}
    for fp64 in (False, True):
        ll = np.frombuffer(raw, dtype=np.float64, count=F, offset=o)
        o += 8 * F
        nr = np.frombuffer(raw, dtype=np.uint32, count=F, offset=o)
        o += 4 * F
        got[fp64] = (ll, nr)
    for fp64 in (False, True):
        assert np.array_equal(got[fp64][1], want[fp64][1]), fp64
        assert np.array_equal(got[fp64][0].view(np.uint64), want[fp64][0].view(np.uint64)), (
            fp64, got[fp64][0][:4], want[fp64][0][:4])
    assert want[False][1].sum() > 0  # the filters resampled
