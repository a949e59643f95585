"""mckl_b200 -- B200 (sm_100a) implementation of MCKL's counter-based RNG,
distribution and SMC hot path, reached through the C ABI in
``include/mckl_b200.h`` (library ``mckl_b200/libmckl_b200.so``).

The Python layer mirrors the reference's interface so tests and benchmarks
read like the reference's own code:

* engines: :class:`Philox4x32`, :class:`Threefry4x64`, :class:`ARS` and the
  ``_64`` variants (``mckl::CounterEngine``, random/counter.hpp:61-288) with
  ``seed`` / ``key`` / ``ctr`` / ``discard``;
* ``rand(rng, n, r)`` and the batch distributions
  ``u01_*_distribution``, ``normal_distribution``,
  ``exponential_distribution``, ``gamma_distribution``
  (random/internal/common.hpp:69-151);
* SMC: ``Weight`` (core/weight.hpp), the resampling schemes
  (algorithm/resample.hpp) and the AR(1) particle filters.

Device memory and streams come from PyTorch tensors; the arithmetic is the
library's own CUDA.  There is no CPU fallback: importing this package on a
machine without the built library raises, and calls without a GPU fail.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmckl_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing; build it with `python mckl_b200/build.py` (nvcc, sm_100a)")

_lib = ctypes.CDLL(LIB_PATH)

PHILOX4X32, PHILOX4X32_64, THREEFRY4X64, THREEFRY4X64_64, ARS_KIND, ARS_64_KIND = range(1, 7)
_WORDS = {1: 4, 2: 2, 3: 8, 4: 4, 5: 4, 6: 2}
_RESULT_BITS = {1: 32, 2: 64, 3: 32, 4: 64, 5: 32, 6: 64}


class MCKLB200Error(RuntimeError):
    pass


class EngineState(ctypes.Structure):
    """``mckl_b200_engine_t``."""

    _fields_ = [
        ("ctr", ctypes.c_uint64 * 4),
        ("key", ctypes.c_uint64 * 4),
        ("tweak", ctypes.c_uint64 * 2),
        ("index", ctypes.c_uint32),
        ("kind", ctypes.c_uint32),
    ]


_vp, _sz, _i, _u32, _u64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64
_f, _d = ctypes.c_float, ctypes.c_double
_EP = ctypes.POINTER(EngineState)


def _bind(name, argtypes, restype=ctypes.c_int):
    fn = getattr(_lib, name)
    fn.argtypes = argtypes
    fn.restype = restype
    return fn


_lib.mckl_b200_last_error.restype = ctypes.c_char_p
_lib.mckl_b200_version.restype = ctypes.c_char_p
_lib.mckl_b200_launch_count.restype = ctypes.c_uint64
_engine_seed = _bind("mckl_b200_engine_seed", [_EP, _u32, _u64])
_engine_discard = _bind("mckl_b200_engine_discard", [_EP, _u64])
_rand = _bind("mckl_b200_rand", [_EP, _sz, _vp, _vp])
_philox_kernel = _bind("mckl_b200_philox4x32_kernel", [_vp, _sz, _vp, _vp, _vp])
_threefry_kernel = _bind("mckl_b200_threefry4x64_kernel", [_vp, _sz, _vp, _vp, _vp, _vp])
_ars_kernel = _bind("mckl_b200_ars_kernel", [_vp, _sz, _vp, _vp, _vp])
_u01 = {}
for _name in ("canonical", "cc", "co", "oc", "oo"):
    for _t in ("f32", "f64"):
        _u01[(_name, _t)] = _bind(f"mckl_b200_u01_{_name}_{_t}", [_EP, _sz, _vp, _vp])
_normal = {"f32": _bind("mckl_b200_normal_f32", [_EP, _sz, _vp, _f, _f, _vp]),
           "f64": _bind("mckl_b200_normal_f64", [_EP, _sz, _vp, _d, _d, _vp])}
_exponential = {"f32": _bind("mckl_b200_exponential_f32", [_EP, _sz, _vp, _f, _vp]),
                "f64": _bind("mckl_b200_exponential_f64", [_EP, _sz, _vp, _d, _vp])}
_gamma = {"f32": _bind("mckl_b200_gamma_f32", [_EP, _sz, _vp, _f, _f, _vp]),
          "f64": _bind("mckl_b200_gamma_f64", [_EP, _sz, _vp, _d, _d, _vp])}
_engine_save = _bind("mckl_b200_engine_save", [_EP, ctypes.c_char_p, _sz, ctypes.POINTER(_sz)])
_engine_load = _bind("mckl_b200_engine_load", [_EP, _u32, ctypes.c_char_p])
_gamma_blocks = {"f32": _bind("mckl_b200_gamma_blocks_f32", [_EP, _sz, _sz, _vp, _d, _vp, _vp]),
                 "f64": _bind("mckl_b200_gamma_blocks_f64", [_EP, _sz, _sz, _vp, _d, _vp, _vp])}


_math_f64 = _bind("mckl_b200_math_f64", [_i, _sz, _vp, _vp, _vp, _vp])


def math_f64(fn: str, x):
    """The library's double-double log / exp / sincos on a CUDA float64 tensor."""
    torch = _torch()
    code = {"log": 0, "exp": 1, "sincos": 2}[fn]
    y = torch.empty_like(x)
    y2 = torch.empty_like(x) if code == 2 else None
    _check(_math_f64(code, x.numel(), ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                     ctypes.c_void_p(y2.data_ptr()) if y2 is not None else None, _stream_ptr()))
    return (y, y2) if code == 2 else y


_weight_set_log = _bind("mckl_b200_weight_set_log", [_sz, _vp, _vp, _vp, _vp, _vp])
_weight_add_log = _bind("mckl_b200_weight_add_log", [_sz, _vp, _vp, _vp, _vp, _vp])
_fold_f64 = _bind("mckl_b200_fold_f64", [_sz, _vp, _d, _vp, _vp, _vp])


_u01_sequence = _bind("mckl_b200_u01_sequence", [_i, _EP, _sz, _vp, _vp])
_resample = _bind("mckl_b200_resample", [_i, _sz, _sz, _EP, _vp, _vp, _vp])
_rep_to_index = _bind("mckl_b200_rep_to_index", [_sz, _sz, _vp, _vp, _vp])
_select = {"f64": _bind("mckl_b200_select_f64", [_sz, _sz, _vp, _vp, _vp]),
           "f32": _bind("mckl_b200_select_f32", [_sz, _sz, _vp, _vp, _vp])}

Multinomial, Stratified, Systematic, Residual, ResidualStratified, ResidualSystematic = range(6)


def u01_sequence(kind: int, rng: CounterEngine, n: int):
    """kind 0 sorted, 1 stratified, 2 systematic (algorithm/resample.hpp:216-268)."""
    torch = _torch()
    u = torch.empty(max(n, 1), dtype=torch.float64, device="cuda")
    _check(_u01_sequence(kind, ctypes.byref(rng.state), n, ctypes.c_void_p(u.data_ptr()), _stream_ptr()))
    return u[:n]


def resample(scheme: int, rng: CounterEngine, W, M=None):
    """Replication counts: ResampleAlgorithm::operator()(N, M, rng, W, rep)."""
    torch = _torch()
    N = W.numel()
    M = N if M is None else M
    rep = torch.empty(N, dtype=torch.int64, device=W.device)
    _check(_resample(scheme, N, M, ctypes.byref(rng.state), ctypes.c_void_p(W.data_ptr()),
                     ctypes.c_void_p(rep.data_ptr()), _stream_ptr()))
    return rep


def rep_to_index(rep, M=None):
    torch = _torch()
    N = rep.numel()
    M = int(rep.sum().item()) if M is None else M
    idx = torch.empty(max(M, 1), dtype=torch.int64, device=rep.device)
    _check(_rep_to_index(N, M, ctypes.c_void_p(rep.data_ptr()), ctypes.c_void_p(idx.data_ptr()), _stream_ptr()))
    return idx[:M]


def select(idx, state):
    """In-place row selection of an N x dim column-major state (dim-major tensor [dim, N] or [N])."""
    torch = _torch()
    N = state.shape[-1]
    dim = state.numel() // N
    t = "f64" if state.dtype == torch.float64 else "f32"
    _check(_select[t](N, dim, ctypes.c_void_p(idx.data_ptr()), ctypes.c_void_p(state.data_ptr()), _stream_ptr()))
    return state


_pf_plain = _bind("mckl_b200_pf_ar1_plain_f64", [_sz, _sz, _vp, _d, _d, _d, _d, _vp, _vp, _i, _d, _vp, _vp,
                                                   _vp, _vp, _vp, _vp, _vp])
_pf_plain_ties = _bind("mckl_b200_pf_ar1_plain_ties", [ctypes.POINTER(ctypes.c_uint64)])


def pf_ar1_plain(N, y, phi, sx, sy, sd0, mkey, rkey, scheme=2, threshold=0.5, record=False):
    """Plain FP64 bootstrap particle filter (see mckl_b200_pf_ar1_plain_f64)."""
    torch = _torch()
    y = np.ascontiguousarray(y, dtype=np.float64)
    T = len(y) - 1
    mk = (ctypes.c_uint32 * 2)(*[int(k) for k in mkey])
    rk = (ctypes.c_uint32 * 2)(*[int(k) for k in rkey])
    ll = ctypes.c_double()
    ess = np.zeros(T + 1)
    rs = np.zeros(T + 1, dtype=np.uint8)
    anc = torch.zeros((T + 1, N), dtype=torch.int64, device="cuda") if record else None
    x = torch.empty(N, dtype=torch.float64, device="cuda")
    W = torch.empty(N, dtype=torch.float64, device="cuda")
    _check(_pf_plain(N, T, y.ctypes.data_as(ctypes.c_void_p), phi, sx, sy, sd0, ctypes.cast(mk, _vp),
                     ctypes.cast(rk, _vp), scheme, threshold, ctypes.byref(ll), ess.ctypes.data_as(ctypes.c_void_p),
                     rs.ctypes.data_as(ctypes.c_void_p),
                     ctypes.c_void_p(anc.data_ptr()) if anc is not None else None,
                     ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(W.data_ptr()), _stream_ptr()))
    ties = ctypes.c_uint64()
    _check(_pf_plain_ties(ctypes.byref(ties)))
    return dict(loglik=ll.value, ess=ess, resampled=rs, anc=anc, x=x, W=W, ties=int(ties.value))


_bt_create = _bind("mckl_b200_batched_create", [_vp, _sz, _vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _d, _i])
_bt_config = _bind("mckl_b200_batched_config", [_vp, _i, _i])
_bt_run = _bind("mckl_b200_batched_run", [_vp, _vp])
_bt_run_graph = _bind("mckl_b200_batched_run_graph", [_vp, _vp])
_bt_results = _bind("mckl_b200_batched_results", [_vp, _vp, _vp, _vp])
_bt_destroy = _bind("mckl_b200_batched_destroy", [_vp])
_bt_shadow = _bind("mckl_b200_batched_shadow", [_vp, _vp, _vp])
_bt_set_y = _bind("mckl_b200_batched_set_y", [_vp, _vp, _vp])
_bt_autotune = _bind("mckl_b200_batched_autotune", [_vp, _i, _vp, _vp, _vp, _vp, _vp])
_bt_get_config = _bind("mckl_b200_batched_get_config", [_vp, _vp, _vp])
_bt_shadow_params = _bind("mckl_b200_batched_shadow_params", [_vp, _vp, _vp, _vp])
_bt_adjoint = _bind("mckl_b200_batched_adjoint", [_vp, _i, _vp, _vp, _vp])
_bt_score = _bind("mckl_b200_batched_score", [_vp, _vp, _vp, _vp])
_bt_set_params = _bind("mckl_b200_batched_set_params", [_vp, _vp, _vp, _vp, _vp])
_bt_set_keys = _bind("mckl_b200_batched_set_keys", [_vp, _vp, _vp, _vp])
_LOG_PRIOR = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)
_pmcmc = _bind("mckl_b200_pmcmc_ar1", [_sz, _vp, _sz, _vp, _vp, _vp, _LOG_PRIOR, _vp, _sz, ctypes.c_uint32, _i,
                                       _d, _vp, _vp, _vp, _vp])
_PROPOSAL = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_size_t, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint32),
                             ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)
_pmcmc_prop = _bind("mckl_b200_pmcmc_ar1_proposal", [_sz, _vp, _sz, _vp, _vp, _PROPOSAL, _vp, _LOG_PRIOR, _vp, _sz,
                                                     ctypes.c_uint32, _i, _d, _vp, _vp, _vp, _vp])


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class BatchedFilters:
    """Many independent AR(1) bootstrap filters in one persistent kernel
    (mckl_b200_batched_*).  y: array [F, T + 1]; keys: arrays [F, 2]."""

    def __init__(self, N, y, phi, sx, sy, mkeys, rkeys, threshold=0.5, fp64=False, shadow=False):
        self.N = _arr(N, np.uint64)
        self.y = _arr(y, np.float64)
        self.F, T1 = self.y.shape
        self.T = T1 - 1
        self._keep = [self.N, self.y, _arr(phi, np.float64), _arr(sx, np.float64), _arr(sy, np.float64),
                      _arr(mkeys, np.uint32), _arr(rkeys, np.uint32)]
        h = ctypes.c_void_p()
        ptrs = [a.ctypes.data_as(ctypes.c_void_p) for a in self._keep]
        mode = (3 if fp64 else 2) if shadow else int(bool(fp64))
        _check(_bt_create(ctypes.byref(h), self.F, ptrs[0], self.T, ptrs[1], ptrs[2], ptrs[3], ptrs[4], ptrs[5],
                          ptrs[6], threshold, mode))
        self.h = h

    def config(self, threads=256, ctas_per_sm=4):
        _check(_bt_config(self.h, threads, ctas_per_sm))

    def run(self, graph=False, stream=None):
        _check((_bt_run_graph if graph else _bt_run)(self.h, _stream_ptr(stream)))

    def results(self):
        ll = np.zeros(self.F)
        nr = np.zeros(self.F, dtype=np.uint32)
        _check(_bt_results(self.h, ll.ctypes.data_as(ctypes.c_void_p), nr.ctypes.data_as(ctypes.c_void_p),
                           _stream_ptr()))
        return ll, nr

    def autotune(self, stream=None):
        """Time the candidate block shapes on these filters and keep the
        fastest; returns [(threads, ctas_per_sm, ms), ...].  A workload tuned
        before in this process is configured from the kept pick without
        timing: then the one entry is that pick with ms = nan."""
        th = (ctypes.c_int * 16)()
        cp = (ctypes.c_int * 16)()
        ms = (ctypes.c_float * 16)()
        n = ctypes.c_int()
        _check(_bt_autotune(self.h, 16, th, cp, ms, ctypes.byref(n), _stream_ptr(stream)))
        if n.value == 0:
            return [self.shape() + (float("nan"),)]
        return [(th[k], cp[k], ms[k]) for k in range(min(n.value, 16))]

    def shape(self):
        """(threads per CTA, resident CTAs per SM) the handle runs with."""
        t, c = ctypes.c_int(), ctypes.c_int()
        _check(_bt_get_config(self.h, ctypes.byref(t), ctypes.byref(c)))
        return (t.value, c.value)

    def set_shadow_params(self, phi, sx, sy):
        """Parameters of the FP64 shadow (handles made with shadow=True)."""
        a = [_arr(v, np.float64) for v in (phi, sx, sy)]
        _check(_bt_shadow_params(self.h, *[v.ctypes.data_as(ctypes.c_void_p) for v in a]))

    def adjoint(self, checkpoint_every=32, stream=None):
        """(loglik[F], grad[F, 3]): the FP64 estimate and its gradient with
        respect to (phi, sx, sy), ancestors held fixed (fp64=True handles)."""
        ll = np.zeros(self.F)
        g = np.zeros((self.F, 3))
        _check(_bt_adjoint(self.h, int(checkpoint_every), ll.ctypes.data_as(ctypes.c_void_p),
                           g.ctypes.data_as(ctypes.c_void_p), _stream_ptr(stream)))
        return ll, g

    def score(self, stream=None):
        """(loglik[F], score[F, 3]): the FP64 estimate and a consistent
        estimate of the score d log p(y | theta) / d (phi, sx, sy) by the
        Fisher identity (PaRIS smoothing in the same pass; fp64=True handles)."""
        ll = np.zeros(self.F)
        g = np.zeros((self.F, 3))
        _check(_bt_score(self.h, ll.ctypes.data_as(ctypes.c_void_p), g.ctypes.data_as(ctypes.c_void_p),
                         _stream_ptr(stream)))
        return ll, g

    def set_params(self, phi, sx, sy, stream=None):
        """New (phi, sx, sy) for every filter; the next run uses them."""
        a = [_arr(v, np.float64) for v in (phi, sx, sy)]
        _check(_bt_set_params(self.h, *[v.ctypes.data_as(ctypes.c_void_p) for v in a], _stream_ptr(stream)))

    def set_keys(self, mkeys, rkeys, stream=None):
        """New model / resampling keys ([F, 2] each) for every filter."""
        m, r = _arr(mkeys, np.uint32), _arr(rkeys, np.uint32)
        _check(_bt_set_keys(self.h, m.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p),
                            _stream_ptr(stream)))

    def set_y(self, y, stream=None):
        """Copy new observations (host array [F, T + 1]; page-locked for an async copy)."""
        ptr = y.data_ptr() if hasattr(y, "data_ptr") else np.ascontiguousarray(y, dtype=np.float64).ctypes.data
        _check(_bt_set_y(self.h, ctypes.c_void_p(ptr), _stream_ptr(stream)))

    def shadow_loglik(self):
        """FP64 log-likelihoods along the FP32 run's genealogy (shadow=True)."""
        ll = np.zeros(self.F)
        _check(_bt_shadow(self.h, ll.ctypes.data_as(ctypes.c_void_p), _stream_ptr()))
        return ll

    def close(self):
        if getattr(self, "h", None):
            _bt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may already be gone
            pass


def batched_workload(F=4096, T=500, seed=1234, nmin=256, nmax=65536, first=0):
    """The batched configuration, filters first .. first + F - 1 of it: filter
    parameters from Philox4x32(seed) canonical uniforms, four per filter in
    filter order (phi ~ U[0.5, 0.99], sx ~ U[0.5, 2], sy ~ U[0.2, 1],
    N = round(exp(U[ln nmin, ln nmax]))), observations of filter f simulated
    with Philox4x32(key f, 10) (2T + 2 standard normals: x_0 = sd0 z_0,
    x_t = phi x_{t-1} + sx z_t, y_t = x_t + sy z_{T+t}); model keys (f, 11),
    resampling keys (f, 12).  A rank of a multi-GPU run takes its own range
    of filters (mckl_b200.shard.filter_range)."""
    torch = _torch()
    g = Philox4x32()
    g.key = (seed, 0)
    u = u01_canonical_distribution(g, 4 * (first + F), dtype="f64").cpu().numpy().reshape(first + F, 4)[first:]
    phi = 0.5 + 0.49 * u[:, 0]
    sx = 0.5 + 1.5 * u[:, 1]
    sy = 0.2 + 0.8 * u[:, 2]
    N = np.rint(np.exp(np.log(nmin) + (np.log(nmax) - np.log(nmin)) * u[:, 3])).astype(np.uint64)
    z = torch.empty((F, 2 * T + 2), dtype=torch.float64, device="cuda")
    for f in range(F):
        gf = Philox4x32()
        gf.key = (first + f, 10)
        normal_distribution(gf, 2 * T + 2, z[f])
    z = z.cpu().numpy()
    sd0 = sx / np.sqrt(1 - phi * phi)
    x = sd0 * z[:, 0]
    y = np.zeros((F, T + 1))
    for t in range(1, T + 1):
        x = phi * x + sx * z[:, t]
        y[:, t] = x + sy * z[:, T + t]
    ids = np.arange(first, first + F)
    mkeys = np.stack([ids, np.full(F, 11)], axis=1).astype(np.uint32)
    rkeys = np.stack([ids, np.full(F, 12)], axis=1).astype(np.uint32)
    return dict(N=N, y=y, phi=phi, sx=sx, sy=sy, sd0=sd0, mkeys=mkeys, rkeys=rkeys)


_index_matrix = _bind("mckl_b200_index_matrix", [_sz, _sz, _vp, _vp, _i, _vp, _vp])
_west = _bind("mckl_b200_weighted_estimate", [_sz, _sz, _i, _vp, _vp, _vp, _vp])


def weighted_estimate(u, W, col_major=False):
    """SMCEstimator's estimate: sum_i W_i u[i, :] (u: CUDA float64 [n, d],
    or [d, n] with col_major)."""
    torch = _torch()
    u = u.contiguous()
    n = W.numel()
    if u.dim() == 2:
        d = u.shape[0] if col_major else u.shape[1]
    else:
        d = u.numel() // max(n, 1)
    if u.numel() != n * d or u.dtype != torch.float64 or W.dtype != torch.float64:
        raise ValueError("u: float64 [n, d] (or [d, n] with col_major), W: float64 [n]")
    out = torch.empty(d, dtype=torch.float64, device="cuda")
    _check(_west(n, d, int(bool(col_major)), ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(W.data_ptr()),
                 ctypes.c_void_p(out.data_ptr()), _stream_ptr()))
    return out


class ResampleIndex:
    """mckl::ResampleIndex over parent-index vectors kept in device memory
    (algorithm/resample.hpp:597-832): push_back, index, index_matrix."""

    RowMajor, ColMajor = 0, 1

    def __init__(self):
        self._v = []
        self._ptr = []  # device addresses and sizes of the vectors, kept beside them
        self._len = []
        self._arrays = {}  # (first, last) -> ctypes address / size arrays of that range

    def num_iter(self):
        return len(self._v)

    def size(self, iter_=None):
        if not self._v:
            return 0
        return int(self._v[-1 if iter_ is None else iter_].numel())

    def reset(self):
        self._v = []
        self._ptr = []
        self._len = []
        self._arrays = {}

    def push_back(self, N, index=None):
        """Append the parent indices of one iteration (a CUDA int64/uint64
        tensor of N entries), or the identity when `index` is None."""
        torch = _torch()
        if index is None:
            index = torch.arange(N, dtype=torch.int64, device="cuda")
        if index.numel() != N or not index.is_cuda or index.element_size() != 8:
            raise ValueError("index: CUDA tensor of N 64-bit integers")
        v = index.contiguous()
        self._v.append(v)
        self._ptr.append(v.data_ptr())
        self._len.append(v.numel())

    def _run(self, rows, col_major):
        """rows: the vector numbers, oldest first (the last is the one whose
        particles the result describes)."""
        torch = _torch()
        key = tuple(rows)
        arr = self._arrays.get(key)
        if arr is None:
            arr = ((ctypes.c_uint64 * len(rows))(*[self._ptr[r] for r in rows]),
                   (ctypes.c_size_t * len(rows))(*[self._len[r] for r in rows]))
            self._arrays = {key: arr}  # one range kept: the usual caller repeats it
        R = len(rows)
        N = int(self._len[rows[-1]])
        out = torch.empty(N * R, dtype=torch.int64, device="cuda")
        _check(_index_matrix(N, R, ctypes.cast(arr[0], _vp), ctypes.cast(arr[1], _vp), int(col_major),
                             ctypes.c_void_p(out.data_ptr()), _stream_ptr()))
        return out

    def index_matrix(self, layout=0, iter_back=None, iter_=0):
        """N x R ancestors (flattened, row- or column-major) of iterations
        iter_..iter_back, N the size at iter_back (:718-829)."""
        ib = self.num_iter() - 1 if iter_back is None else iter_back
        if not (0 <= iter_ <= ib < self.num_iter()):
            raise IndexError("iteration numbers out of range")
        return self._run(list(range(iter_, ib + 1)), layout == self.ColMajor)

    def index(self, id_, iter_back=None, iter_=0):
        """index(id, iter_back, iter) (:666-678): from the last iteration's
        vector, followed back through iterations iter_back - 1 .. iter_."""
        ib = self.num_iter() - 1 if iter_back is None else iter_back
        if not (0 <= iter_ <= ib < self.num_iter()):
            raise IndexError("iteration numbers out of range")
        col = self._run(list(range(iter_, ib)) + [self.num_iter() - 1], True)
        return int(col[id_].item())


def pmcmc_ar1(y, N, theta0, step, log_prior, iters, seed=1, fp64=False, threshold=0.5, proposal=None):
    """Particle marginal Metropolis-Hastings, C chains at once
    (mckl_b200_pmcmc_ar1).  y: [C, T + 1] (or [T + 1], shared); N: particles
    per chain (int or [C]); theta0: [C, 3] = (phi, sx, sy); step: random-walk
    scales [3]; log_prior(theta) -> float.  `proposal(chain, iteration,
    words, theta)`, when given, replaces the random walk
    (mckl_b200_pmcmc_ar1_proposal, PMCMCMutation's update evaluations): it
    changes theta (a float64 array of 3) in place from the four uint32 words
    and returns the log proposal ratio log q(theta | theta') -
    log q(theta' | theta).  Returns (theta [iters, C, 3], loglik [iters, C],
    accepted [C])."""
    theta0 = _arr(np.atleast_2d(theta0), np.float64)
    C = theta0.shape[0]
    y = np.asarray(y, dtype=np.float64)
    if y.ndim == 1:
        y = np.broadcast_to(y, (C, y.shape[0]))
    y = _arr(y, np.float64)
    T = y.shape[1] - 1
    Nv = _arr(np.broadcast_to(np.asarray(N, dtype=np.uint64), (C,)), np.uint64)
    st = _arr(step, np.float64)
    th = np.zeros((iters, C, 3))
    ll = np.zeros((iters, C))
    acc = np.zeros(C, dtype=np.uint32)

    def _prior(p, _user):
        return float(log_prior(np.array([p[0], p[1], p[2]])))

    cb = _LOG_PRIOR(_prior)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    if proposal is None:
        _check(_pmcmc(C, vp(Nv), T, vp(y), vp(theta0), vp(st), cb, None, iters, seed & 0xFFFFFFFF,
                      int(bool(fp64)), threshold, vp(th), vp(ll), vp(acc), _stream_ptr()))
        return th, ll, acc

    def _prop(chain, it, words, theta, _user):
        w = np.array([words[k] for k in range(4)], dtype=np.uint32)
        t = np.ctypeslib.as_array(theta, shape=(3,))
        return float(proposal(int(chain), int(it), w, t))

    pcb = _PROPOSAL(_prop)
    _check(_pmcmc_prop(C, vp(Nv), T, vp(y), vp(theta0), pcb, None, cb, None, iters, seed & 0xFFFFFFFF,
                       int(bool(fp64)), threshold, vp(th), vp(ll), vp(acc), _stream_ptr()))
    return th, ll, acc


def fold_f64(x, s0: float = 0.0, prefix=True):
    """Exact emulation of the sequential left fold; returns (prefix tensor or None, final)."""
    torch = _torch()
    pre = torch.empty_like(x) if prefix else None
    fin = ctypes.c_double()
    _check(_fold_f64(x.numel(), ctypes.c_void_p(x.data_ptr()), s0,
                     ctypes.c_void_p(pre.data_ptr()) if pre is not None else None, ctypes.byref(fin),
                     _stream_ptr()))
    return pre, fin.value


class Weight:
    """``mckl::Weight`` over a CUDA float64 tensor of normalised weights."""

    def __init__(self, N: int, device="cuda"):
        torch = _torch()
        self.data = torch.full((N,), 1.0 / N, dtype=torch.float64, device=device)
        self._ess = float(N)
        self.log_nc = 0.0

    def size(self) -> int:
        return self.data.numel()

    def ess(self) -> float:
        return self._ess

    def set_equal(self) -> None:
        self.data.fill_(1.0 / self.size())
        self._ess = float(self.size())

    def _call(self, fn, v):
        torch = _torch()
        v = v.to(device=self.data.device, dtype=torch.float64).contiguous()
        ess, lnc = ctypes.c_double(), ctypes.c_double()
        _check(fn(self.size(), ctypes.c_void_p(self.data.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                  ctypes.byref(ess), ctypes.byref(lnc), _stream_ptr()))
        self._ess = ess.value
        self.log_nc = lnc.value

    def set_log(self, v) -> None:
        self._call(_weight_set_log, v)

    def add_log(self, v) -> None:
        self._call(_weight_add_log, v)


def _check(rc: int) -> None:
    if rc != 0:
        raise MCKLB200Error(f"mckl_b200 error {rc}: {_lib.mckl_b200_last_error().decode()}")


def version() -> str:
    return _lib.mckl_b200_version().decode()


def launch_count() -> int:
    """Kernels launched by the library so far in this process."""
    return int(_lib.mckl_b200_launch_count())


def lib_path() -> str:
    return LIB_PATH


def raw_lib() -> ctypes.CDLL:
    """The loaded C-ABI library (for callers binding further entry points)."""
    return _lib


# ---------------------------------------------------------------------------
# engines
# ---------------------------------------------------------------------------
class CounterEngine:
    """Host handle of one counter-based engine (``mckl::CounterEngine``).

    The state lives on the host and is advanced by every call exactly as the
    reference engine's would be; the words themselves are produced on the GPU.
    """

    kind = 0

    def __init__(self, seed: int = 1, key=None):
        self.state = EngineState()
        self.seed(seed)
        if key is not None:
            self.key = key

    # -- reference API ----------------------------------------------------
    def seed(self, s: int) -> None:
        _check(_engine_seed(ctypes.byref(self.state), self.kind, int(s)))

    @property
    def key(self):
        n = 2 if self.kind in (PHILOX4X32, PHILOX4X32_64) else 4
        return tuple(int(self.state.key[i]) for i in range(n))

    @key.setter
    def key(self, k) -> None:
        # CounterEngine::key(k) == seed(k): counter reset, nothing buffered
        for i in range(4):
            self.state.key[i] = int(k[i]) if i < len(k) else 0
        for i in range(4):
            self.state.ctr[i] = 0
        self.state.index = _WORDS[self.kind]

    @property
    def ctr(self):
        n = 4 if self.kind in (THREEFRY4X64, THREEFRY4X64_64) else 2
        return tuple(int(self.state.ctr[i]) for i in range(n))

    @ctr.setter
    def ctr(self, c) -> None:
        # CounterEngine::ctr(c): set the counter, drop the buffer (random/counter.hpp:129-133)
        for i in range(4):
            self.state.ctr[i] = int(c[i]) if i < len(c) else 0
        self.state.index = _WORDS[self.kind]

    @property
    def index(self) -> int:
        return int(self.state.index)

    def discard(self, nskip: int) -> None:
        _check(_engine_discard(ctypes.byref(self.state), int(nskip)))

    def words_per_block(self) -> int:
        return _WORDS[self.kind]

    def result_bits(self) -> int:
        return _RESULT_BITS[self.kind]

    def copy(self):
        other = type(self).__new__(type(self))
        other.state = EngineState()
        ctypes.pointer(other.state)[0] = self.state
        return other

    def state_tuple(self):
        s = self.state
        return (tuple(s.ctr), tuple(s.key), tuple(s.tweak), int(s.index), int(s.kind))

    def __str__(self) -> str:
        """The reference's ``os << rng`` text (random/counter.hpp:235-252)."""
        n = _sz()
        _check(_engine_save(ctypes.byref(self.state), None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        _check(_engine_save(ctypes.byref(self.state), buf, n.value + 1, ctypes.byref(n)))
        return buf.value.decode()

    def load_text(self, text: str) -> None:
        """The reference's ``is >> rng`` (random/counter.hpp:254-272); raises
        on text that is not a state of this engine kind."""
        _check(_engine_load(ctypes.byref(self.state), self.kind, text.encode()))

    @classmethod
    def from_text(cls, text: str):
        e = cls.__new__(cls)
        e.state = EngineState()
        e.load_text(text)
        return e

    def load_state(self, ctr, key, tweak, index) -> None:
        for i in range(4):
            self.state.ctr[i] = int(ctr[i])
            self.state.key[i] = int(key[i])
        self.state.tweak[0], self.state.tweak[1] = int(tweak[0]), int(tweak[1])
        self.state.index = int(index)


class Philox4x32(CounterEngine):
    kind = PHILOX4X32


class Philox4x32_64(CounterEngine):
    kind = PHILOX4X32_64


class Threefry4x64(CounterEngine):
    kind = THREEFRY4X64

    def tweak(self, t0: int, t1: int) -> None:
        self.state.tweak[0], self.state.tweak[1] = int(t0), int(t1)


class Threefry4x64_64(Threefry4x64):
    kind = THREEFRY4X64_64


class ARS(CounterEngine):
    kind = ARS_KIND


class ARS_64(CounterEngine):
    kind = ARS_64_KIND


ENGINES = {"Philox4x32": Philox4x32, "Philox4x32_64": Philox4x32_64, "Threefry4x64": Threefry4x64,
           "Threefry4x64_64": Threefry4x64_64, "ARS": ARS, "ARS_64": ARS_64}


# ---------------------------------------------------------------------------
# tensors and streams
# ---------------------------------------------------------------------------
def _torch():
    import torch  # local: the library itself does not need torch

    return torch


def _stream_ptr(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _check_out(r, n: int, itemsize: int):
    torch = _torch()
    if not isinstance(r, torch.Tensor) or not (r.is_cuda or r.is_pinned()):
        raise MCKLB200Error("output must be a CUDA tensor or a pinned host tensor")
    if not r.is_contiguous() or r.element_size() != itemsize or r.numel() < n:
        raise MCKLB200Error("output tensor has the wrong size, dtype width or layout")
    return ctypes.c_void_p(r.data_ptr())


def empty_words(rng: CounterEngine, n: int, device="cuda"):
    torch = _torch()
    return torch.empty(n, dtype=torch.int64 if rng.result_bits() == 64 else torch.int32, device=device)


# ---------------------------------------------------------------------------
# RNG and distributions (reference batch calls)
# ---------------------------------------------------------------------------
def rand(rng: CounterEngine, n: int, r=None, stream=None):
    """``mckl::rand(rng, n, r)``: n raw result words (int32/int64 tensor bits)."""
    if r is None:
        r = empty_words(rng, n)
    ptr = _check_out(r, n, rng.result_bits() // 8)
    _check(_rand(ctypes.byref(rng.state), n, ptr, _stream_ptr(stream)))
    return r


def _real_out(r, n, dtype):
    torch = _torch()
    if r is None:
        r = torch.empty(n, dtype=torch.float64 if dtype == "f64" else torch.float32, device="cuda")
    t = "f64" if r.dtype == torch.float64 else "f32"
    if t != dtype and dtype is not None:
        raise MCKLB200Error("output dtype mismatch")
    return r, t


def _u01_call(variant, rng, n, r, dtype, stream):
    r, t = _real_out(r, n, dtype)
    ptr = _check_out(r, n, 8 if t == "f64" else 4)
    _check(_u01[(variant, t)](ctypes.byref(rng.state), n, ptr, _stream_ptr(stream)))
    return r


def u01_canonical_distribution(rng, n, r=None, dtype="f64", stream=None):
    return _u01_call("canonical", rng, n, r, None if r is not None else dtype, stream)


u01_distribution = u01_canonical_distribution


def u01_cc_distribution(rng, n, r=None, dtype="f64", stream=None):
    return _u01_call("cc", rng, n, r, None if r is not None else dtype, stream)


def u01_co_distribution(rng, n, r=None, dtype="f64", stream=None):
    return _u01_call("co", rng, n, r, None if r is not None else dtype, stream)


def u01_oc_distribution(rng, n, r=None, dtype="f64", stream=None):
    return _u01_call("oc", rng, n, r, None if r is not None else dtype, stream)


def u01_oo_distribution(rng, n, r=None, dtype="f64", stream=None):
    return _u01_call("oo", rng, n, r, None if r is not None else dtype, stream)


def normal_distribution(rng, n, r=None, mean=0.0, stddev=1.0, dtype="f64", stream=None):
    r, t = _real_out(r, n, None if r is not None else dtype)
    ptr = _check_out(r, n, 8 if t == "f64" else 4)
    _check(_normal[t](ctypes.byref(rng.state), n, ptr, mean, stddev, _stream_ptr(stream)))
    return r


def exponential_distribution(rng, n, r=None, lam=1.0, dtype="f64", stream=None):
    r, t = _real_out(r, n, None if r is not None else dtype)
    ptr = _check_out(r, n, 8 if t == "f64" else 4)
    _check(_exponential[t](ctypes.byref(rng.state), n, ptr, lam, _stream_ptr(stream)))
    return r


def gamma_distribution(rng, n, r=None, alpha=1.0, beta=1.0, dtype="f64", stream=None):
    """gamma_distribution(rng, n, r, alpha, beta): one stream, engine advanced."""
    r, t = _real_out(r, n, None if r is not None else dtype)
    ptr = _check_out(r, n, 8 if t == "f64" else 4)
    _check(_gamma[t](ctypes.byref(rng.state), n, ptr, alpha, beta, _stream_ptr(stream)))
    return r


def gamma_blocks(rng, block, alpha, r=None, beta=1.0, dtype="f64", stream=None):
    """Independent Gamma streams: block b = gamma_distribution of `block`
    values with shape alpha[b] from rng positioned at counter (0, b)."""
    alpha = np.ascontiguousarray(alpha, dtype=np.float64)
    n = len(alpha) * block
    r, t = _real_out(r, n, None if r is not None else dtype)
    ptr = _check_out(r, n, 8 if t == "f64" else 4)
    _check(_gamma_blocks[t](ctypes.byref(rng.state), len(alpha), block, alpha.ctypes.data_as(ctypes.c_void_p),
                            beta, ptr, _stream_ptr(stream)))
    return r


def philox4x32_kernel(ctr, n, r, key, stream=None):
    """Generator-level kernel: n blocks for counters ctr+1..ctr+n; returns new ctr."""
    c = (ctypes.c_uint64 * 2)(*[int(x) for x in ctr])
    k = (ctypes.c_uint32 * 2)(*[int(x) for x in key])
    _check(_philox_kernel(ctypes.cast(c, _vp), n, _check_out(r, n * 4, 4), ctypes.cast(k, _vp),
                          _stream_ptr(stream)))
    return (int(c[0]), int(c[1]))


def threefry4x64_kernel(ctr, n, r, key, tweak=(0, 0), stream=None):
    c = (ctypes.c_uint64 * 4)(*[int(x) for x in ctr])
    k = (ctypes.c_uint64 * 4)(*[int(x) for x in key])
    t = (ctypes.c_uint64 * 2)(*[int(x) for x in tweak])
    _check(_threefry_kernel(ctypes.cast(c, _vp), n, _check_out(r, n * 8, 4), ctypes.cast(k, _vp),
                            ctypes.cast(t, _vp), _stream_ptr(stream)))
    return tuple(int(x) for x in c)


def ars_kernel(ctr, n, r, key, stream=None):
    c = (ctypes.c_uint64 * 2)(*[int(x) for x in ctr])
    k = (ctypes.c_uint32 * 4)(*[int(x) for x in key])
    _check(_ars_kernel(ctypes.cast(c, _vp), n, _check_out(r, n * 4, 4), ctypes.cast(k, _vp),
                       _stream_ptr(stream)))
    return (int(c[0]), int(c[1]))


def words_to_numpy(t, bits: int) -> np.ndarray:
    """Copy a device word tensor to a numpy array of unsigned words."""
    a = t.cpu().numpy()
    return a.view(np.uint64 if bits == 64 else np.uint32)
