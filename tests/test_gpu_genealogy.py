"""ResampleIndex trace-back (algorithm/resample.hpp:597-832) on device-resident
parent indices, against the compiled reference's ResampleIndex: random
parent vectors and the genealogy recorded by the plain particle filter;
index matrices in both layouts and sub-ranges of iterations, and the
single-particle trace.  Integer results: bit-identical."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from conftest import require_cuda  # noqa: E402
pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402


@pytest.fixture(scope="module")
def env():
    require_cuda()
    if not O.have_ref():
        pytest.skip("reference build missing")
    import mckl_b200 as mb

    O.build(ref=True)
    return mb, O.CPUPath("ref")


def run(mb, idx, iter_back, iter_, col):
    ri = mb.ResampleIndex()
    for r in range(idx.shape[0]):
        ri.push_back(idx.shape[1], torch.from_numpy(idx[r].astype(np.int64)).cuda())
    m = ri.index_matrix(ri.ColMajor if col else ri.RowMajor, iter_back, iter_).cpu().numpy().astype(np.uint64)
    return ri, m


def test_random_parents(env):
    mb, ref = env
    rng = np.random.default_rng(3)
    N, R = 5000, 17
    idx = rng.integers(0, N, size=(R, N)).astype(np.uint64)
    for (ib, it) in ((R - 1, 0), (R - 1, 5), (R - 1, R - 1)):
        for col in (False, True):
            ri, m = run(mb, idx, ib, it, col)
            want, trace = ref.index_matrix(idx, ib, it, col)
            assert np.array_equal(m, want), (ib, it, col)
        for i in (0, 17, N - 1):
            assert ri.index(i, ib, it) == int(trace[i])
    # iter_back before the last iteration: the reference's index() starts from
    # the last vector, its matrix from iteration iter_back
    ri, m = run(mb, idx, 9, 2, True)
    want, trace = ref.index_matrix(idx, 9, 2, True)
    assert np.array_equal(m, want)
    assert all(ri.index(i, 9, 2) == int(trace[i]) for i in (0, 100, N - 1))


def test_particle_filter_genealogy(env):
    mb, ref = env
    orc = O.CPUPath("oracle")
    N, T = 2048, 40
    y = np.concatenate([[0.0], np.cumsum(np.random.default_rng(1).normal(size=T)) * 0.3])
    r = mb.pf_ar1_plain(N, y, 0.9, 1.0, 0.5, 1.0 / np.sqrt(0.19), (7, 0), (8, 0), record=True)
    anc = r["anc"]  # (T + 1) x N parent indices on the device
    ri = mb.ResampleIndex()
    for t in range(T + 1):
        ri.push_back(N, anc[t])
    m = ri.index_matrix(ri.ColMajor).cpu().numpy().astype(np.uint64)
    want, _ = ref.index_matrix(anc.cpu().numpy().astype(np.uint64), T, 0, True)
    assert np.array_equal(m, want)


def test_bad_parent_rejected(env):
    mb, _ = env
    ri = mb.ResampleIndex()
    ri.push_back(4)
    ri.push_back(8, torch.arange(8, dtype=torch.int64, device="cuda"))  # parents up to 7 > 3
    with pytest.raises(Exception):
        ri.index_matrix()
