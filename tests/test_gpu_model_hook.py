"""The model hook of the batched filters (include/mckl_b200_batched.cuh): a
user's model struct instantiates the persistent kernel in the user's own
translation unit (tests/cpp/batched_model_test.cu, compiled here with nvcc).

* The AR(1) model written as a user would write it (its own struct, the
  explicit roundings of Math<R>), run through mckl_b200::batched_run_model in
  FP32 and FP64: its log-likelihoods and resampling counts equal the
  library's built-in AR(1) filters' (mckl_b200_batched_run) bit for bit, on
  filters of uneven sizes.
* A different model (AR(1) around a mean mu, other arithmetic): one filter of
  2^17 particles, its log-likelihood estimate within Monte Carlo error of the
  exact one (the Kalman filter of y - mu)."""
import os
import subprocess

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    require_cuda()
    d = tmp_path_factory.mktemp("model_hook")
    path = str(d / "batched_model_test")
    r = subprocess.run([os.path.join(CUDA, "bin", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                        "-std=c++17", "--expt-relaxed-constexpr", f"-I{ROOT}/include", f"-I{ROOT}/mckl_b200/csrc",
                        os.path.join(ROOT, "tests", "cpp", "batched_model_test.cu"), "-o", path],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return path, d


def test_user_model_equals_builtin_ar1(exe):
    import mckl_b200 as mb

    path, d = exe
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
    inp, out = str(d / "ar1_in.bin"), str(d / "ar1_out.bin")
    with open(inp, "wb") as f:
        f.write(np.array([F, T], dtype=np.int32).tobytes())
        f.write(np.array([threshold], dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(w["N"], dtype=np.uint64).tobytes())
        for k in ("phi", "sx", "sy"):
            f.write(np.ascontiguousarray(w[k], dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(w["mkeys"], dtype=np.uint32).tobytes())
        f.write(np.ascontiguousarray(w["rkeys"], dtype=np.uint32).tobytes())
        f.write(np.ascontiguousarray(w["y"], dtype=np.float64).tobytes())
    r = subprocess.run([path, "ar1", inp, out], capture_output=True, text=True, timeout=300)
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


def test_other_model_against_kalman(exe):
    from mckl_b200.kalman import kalman_ar1

    path, d = exe
    mu, phi, sx, sy, T, N = 3.0, 0.8, 1.0, 0.6, 100, 1 << 17
    rng = np.random.default_rng(23)
    x = mu + sx / np.sqrt(1 - phi * phi) * rng.normal()
    y = np.zeros(T + 1)
    for t in range(1, T + 1):
        x = mu + phi * (x - mu) + sx * rng.normal()
        y[t] = x + sy * rng.normal()
    inp, out = str(d / "off_in.bin"), str(d / "off_out.bin")
    with open(inp, "wb") as f:
        f.write(np.array([T], dtype=np.int32).tobytes())
        f.write(np.array([5, 11, 5, 12], dtype=np.uint32).tobytes())
        f.write(np.array([N], dtype=np.uint64).tobytes())
        f.write(np.array([mu, phi, sx, sy], dtype=np.float64).tobytes())
        f.write(y.tobytes())
    r = subprocess.run([path, "offset", inp, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = open(out, "rb").read()
    ll = np.frombuffer(raw, dtype=np.float64, count=1)[0]
    nres = np.frombuffer(raw, dtype=np.uint32, count=1, offset=8)[0]
    kf, _ = kalman_ar1(y - mu, phi, sx, sy)
    assert nres > 0
    assert abs(ll - kf[0]) < 0.5, (ll, kf[0])  # Monte Carlo error of 2^17 particles: ~0.05
