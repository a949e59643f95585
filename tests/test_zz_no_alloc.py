"""The allocation-free Weight::add_log entry point.

mckl_b200_weight_add_log_static serves callers that cannot let a library
allocate device memory (a host that owns all device memory through its own
pool, code that must not synchronize the device, processes at the memory
limit).  It keeps its working memory in a fixed array inside the library.
This test calls it through the C ABI and checks it against
mckl_b200_weight_add_log on the same inputs, twice in a row (the second call
finds the first call's leftovers in the shared array), and checks that a
particle count beyond its fixed limit is refused.  It lives in its own file,
collected after the other tests, and passes alone or after them.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    require_cuda()
    import mckl_b200 as mb

    L = mb.raw_lib()
    for name in ("mckl_b200_weight_add_log", "mckl_b200_weight_add_log_static"):
        fn = getattr(L, name)
        fn.argtypes = [ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.c_void_p]
        fn.restype = ctypes.c_int
    return L


def run(fn, W0, v):
    W = W0.clone()
    ess, lnc = ctypes.c_double(), ctypes.c_double()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = fn(W.numel(), ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(v.data_ptr()), ctypes.byref(ess),
            ctypes.byref(lnc), stream)
    return rc, W.cpu().numpy(), ess.value, lnc.value


def test_static_matches_allocating_entry_point(lib):
    rng = np.random.default_rng(2024)
    # the same array serves every size, one after the other; 1 << 22 is the
    # documented maximum, where the working memory nearly fills the array
    for N in (5000, 1 << 20, 1 << 22):
        W0 = rng.random(N)
        W0 /= W0.sum()
        W0 = torch.from_numpy(W0).cuda()
        for call in range(2):
            v = torch.from_numpy(rng.normal(0, 3, N)).cuda()
            rc_a, Wa, ess_a, lnc_a = run(lib.mckl_b200_weight_add_log, W0, v)
            rc_b, Wb, ess_b, lnc_b = run(lib.mckl_b200_weight_add_log_static, W0, v)
            assert rc_a == 0 and rc_b == 0, lib.mckl_b200_last_error()
            # same kernels on the same inputs: identical bits
            assert np.array_equal(Wa.view(np.uint64), Wb.view(np.uint64)), (N, call)
            assert ess_a == ess_b and lnc_a == lnc_b, (N, call)


def test_static_rejects_sizes_beyond_its_limit(lib):
    N = (1 << 22) + 1
    W = torch.full((N,), 1.0 / N, dtype=torch.float64, device="cuda")
    v = torch.zeros(N, dtype=torch.float64, device="cuda")
    rc, _, _, _ = run(lib.mckl_b200_weight_add_log_static, W, v)
    assert rc == -1
    lib.mckl_b200_last_error.restype = ctypes.c_char_p
    assert b"exceeds" in lib.mckl_b200_last_error()
