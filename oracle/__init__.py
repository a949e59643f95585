"""ctypes loader for the CPU checkers (TEST INFRASTRUCTURE ONLY).

Two libraries share one interface:

* ``liboracle.so`` -- the plain-C restatement in ``oracle/oracle.c`` (functions
  ``orc_*``).  It travels with the repository and is what tests, ``smoke()``
  and ``bench.py``'s ``cpu_baseline`` leg compare the CUDA path against.
* ``_ref/libmckl_ref.so`` -- the reference itself, compiled from its own
  headers by ``oracle/Makefile`` (functions ``ref_*``).  Used to pin the
  restatement and to generate ``tests/golden/``; built only where the
  reference sources are present, but once built it travels to the GPU host
  for the ``--impl reference`` timing arm.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU
baseline / reference arm) may import this package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmckl_ref.so")
REF_GENERIC_SO = os.path.join(HERE, "_ref", "libmckl_ref_generic.so")
# The reference's source tree: $MCKL_REF_ROOT, else a `reference` directory
# beside this repository's root.
REF_ROOT = os.environ.get("MCKL_REF_ROOT", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))

PHILOX4X32, PHILOX4X32_64, THREEFRY4X64, THREEFRY4X64_64, ARS, ARS_64 = range(1, 7)
WORDS_PER_BLOCK = {1: 4, 2: 2, 3: 8, 4: 4, 5: 4, 6: 2}
RESULT_DTYPE = {1: np.uint32, 2: np.uint64, 3: np.uint32, 4: np.uint64, 5: np.uint32, 6: np.uint64}
U01_VARIANTS = {"canonical": 0, "cc": 1, "co": 2, "oc": 3, "oo": 4}


class Engine(ctypes.Structure):
    """Counter-engine state; same layout as ``mckl_b200_engine_t``."""

    _fields_ = [
        ("ctr", ctypes.c_uint64 * 4),
        ("key", ctypes.c_uint64 * 4),
        ("tweak", ctypes.c_uint64 * 2),
        ("index", ctypes.c_uint32),
        ("kind", ctypes.c_uint32),
    ]

    @classmethod
    def make(cls, kind, key=(1,), ctr=(0,), index=None, tweak=(0, 0)):
        e = cls()
        e.kind = kind
        for i, k in enumerate(key):
            e.key[i] = int(k)
        for i, c in enumerate(ctr):
            e.ctr[i] = int(c)
        e.tweak[0], e.tweak[1] = int(tweak[0]), int(tweak[1])
        e.index = WORDS_PER_BLOCK[kind] if index is None else int(index)
        return e

    def copy(self):
        e = Engine()
        ctypes.pointer(e)[0] = self
        return e

    def state(self):
        return (tuple(self.ctr), tuple(self.key), tuple(self.tweak), int(self.index), int(self.kind))


def build(ref: bool = False) -> None:
    """Compile the restatement (and, if asked and possible, the reference)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref and os.path.isdir(os.path.join(REF_ROOT, "include", "mckl")):
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)
        if os.path.exists(os.path.join(os.path.dirname(HERE), "mckl_b200", "libmckl_b200.so")):
            subprocess.run(["make", "-s", "-C", HERE, "shim"], check=True)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


class CPUPath:
    """Uniform wrapper over ``orc_*`` (restatement) or ``ref_*`` (reference)."""

    def __init__(self, which: str = "oracle"):
        """which: "oracle" (restatement), "ref" (reference, AES-NI paths on) or
        "ref_generic" (reference with its generic ARS path)."""
        self.which = which
        path = {"oracle": ORACLE_SO, "ref": REF_SO, "ref_generic": REF_GENERIC_SO}[which]
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.p = "orc_" if which == "oracle" else "ref_"
        f = self._f
        sz, vp, i, d = ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        ep = ctypes.POINTER(Engine)
        f("rand", [ep, sz, vp])
        f("u01", [ep, i, i, sz, vp])
        f("normal", [ep, i, sz, vp, d, d])
        f("exponential", [ep, i, sz, vp, d])
        f("gamma", [ep, i, sz, vp, d, d])
        f("gamma_blocks", [ep, i, sz, sz, vp, d, vp, i])
        f("weight_set_log", [sz, vp, vp, vp])
        f("weight_add_log", [sz, vp, vp, vp])
        f("u01_sequence", [i, ep, sz, vp])
        f("u01_trans_sorted", [sz, vp, vp])
        f("rep_to_u01", [sz, sz, vp, vp, vp])
        f("resample", [i, sz, sz, ep, vp, vp])
        f("rep_index", [sz, sz, vp, vp])
        f("select_f64", [sz, sz, vp, vp])
        if which == "oracle":
            f("simulate_ar1", [sz, d, d, d, d, vp, vp, vp])
            f("pf_ar1", [sz, sz, vp, d, d, d, d, vp, vp, i, d, vp, vp, vp, vp, vp, vp])
            f("kalman_ar1", [sz, vp, d, d, d, vp, vp])
            f("block", [ep, vp, vp])
            f("math_f64", [i, sz, vp, vp, vp])
            f("fold", [sz, vp, d, vp, vp])
            f("weighted_estimate", [sz, sz, i, vp, vp, vp])
            f("gamma_blocks_from", [ep, i, sz, sz, sz, vp, d, vp, i])
        else:
            f("pf_ar1", [sz, sz, vp, d, d, d, d, vp, vp, i, d, i, vp, vp, vp, vp, vp, vp, i])
            f("pf_ar1_batch", [sz, vp, sz, vp, vp, vp, vp, vp, vp, i, d, vp, i])
            f("pf_ar1_digest", [sz, sz, vp, d, d, d, d, vp, vp, i, d, vp, vp, vp, vp, vp])
            f("index_matrix", [sz, sz, vp, sz, sz, i, vp, vp])
            f("engine_to_text", [ep, ctypes.c_char_p, sz])
            f("engine_from_text", [ep, ctypes.c_char_p])
            f("engine_text_roundtrip", [ep, ctypes.c_char_p, ctypes.c_char_p, sz])
            f("fill_u32_parallel", [ep, sz, vp, i], restype=d)
            f("dist_parallel", [ep, i, i, sz, vp, i], restype=d)
            f("max_threads", [], restype=i)

    def _f(self, name, argtypes, restype=ctypes.c_int):
        fn = getattr(self.lib, self.p + name)
        fn.argtypes = argtypes
        fn.restype = restype
        setattr(self, "_" + name, fn)

    # -- RNG ---------------------------------------------------------------
    def rand(self, eng: Engine, n: int) -> np.ndarray:
        out = np.zeros(n, dtype=RESULT_DTYPE[eng.kind])
        assert self._rand(ctypes.byref(eng), n, _ptr(out)) == 0
        return out

    def u01(self, eng: Engine, variant: str, f64: bool, n: int) -> np.ndarray:
        out = np.zeros(n, dtype=np.float64 if f64 else np.float32)
        assert self._u01(ctypes.byref(eng), U01_VARIANTS[variant], int(f64), n, _ptr(out)) == 0
        return out

    def normal(self, eng, f64, n, mean=0.0, sd=1.0):
        out = np.zeros(n, dtype=np.float64 if f64 else np.float32)
        assert self._normal(ctypes.byref(eng), int(f64), n, _ptr(out), mean, sd) == 0
        return out

    def exponential(self, eng, f64, n, lam=1.0):
        out = np.zeros(n, dtype=np.float64 if f64 else np.float32)
        assert self._exponential(ctypes.byref(eng), int(f64), n, _ptr(out), lam) == 0
        return out

    def gamma(self, eng, f64, n, alpha, beta=1.0):
        out = np.zeros(n, dtype=np.float64 if f64 else np.float32)
        assert self._gamma(ctypes.byref(eng), int(f64), n, _ptr(out), alpha, beta) == 0
        return out

    def gamma_blocks(self, eng, f64, block, alpha, beta=1.0, nthreads=1):
        alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        out = np.zeros(len(alpha) * block, dtype=np.float64 if f64 else np.float32)
        assert self._gamma_blocks(ctypes.byref(eng), int(f64), len(alpha), block, _ptr(alpha), beta,
                                  _ptr(out), nthreads) == 0
        return out

    def gamma_blocks_from(self, eng, f64, first, block, alpha, beta=1.0, nthreads=1):
        """Blocks first .. first + len(alpha) - 1 of gamma_blocks (oracle only)."""
        alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        out = np.zeros(len(alpha) * block, dtype=np.float64 if f64 else np.float32)
        assert self._gamma_blocks_from(ctypes.byref(eng), int(f64), first, len(alpha), block, _ptr(alpha), beta,
                                       _ptr(out), nthreads) == 0
        return out

    # -- SMC ---------------------------------------------------------------
    def weight_set_log(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        W = np.zeros_like(v)
        ess = np.zeros(1)
        self._weight_set_log(len(v), _ptr(v), _ptr(W), _ptr(ess))
        return W, float(ess[0])

    def weight_add_log(self, W, v):
        W = np.array(W, dtype=np.float64, copy=True)
        v = np.ascontiguousarray(v, dtype=np.float64)
        ess = np.zeros(1)
        self._weight_add_log(len(v), _ptr(W), _ptr(v), _ptr(ess))
        return W, float(ess[0])

    def u01_sequence(self, kind: int, eng, N):
        out = np.zeros(max(N, 1), dtype=np.float64)
        assert self._u01_sequence(kind, ctypes.byref(eng), N, _ptr(out)) == 0
        return out[:N]

    def rep_to_u01(self, W, u):
        W = np.ascontiguousarray(W, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        rep = np.zeros(len(W), dtype=np.uint64)
        self._rep_to_u01(len(W), len(u), _ptr(W), _ptr(u), _ptr(rep))
        return rep

    def resample(self, scheme: int, eng, W, M=None):
        W = np.ascontiguousarray(W, dtype=np.float64)
        N = len(W)
        M = N if M is None else M
        rep = np.zeros(N, dtype=np.uint64)
        assert self._resample(scheme, N, M, ctypes.byref(eng), _ptr(W), _ptr(rep)) == 0
        return rep

    def rep_index(self, rep, M=None):
        rep = np.ascontiguousarray(rep, dtype=np.uint64)
        M = int(rep.sum()) if M is None else M
        idx = np.zeros(max(M, 1), dtype=np.uint64)
        self._rep_index(len(rep), M, _ptr(rep), _ptr(idx))
        return idx[:M]

    def weighted_estimate(self, u, W, col_major=False):
        """SMCEstimator's estimate sum_i W_i u(i, j); u [n, d] (or [d, n]
        with col_major)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        W = np.ascontiguousarray(W, dtype=np.float64)
        n = W.size
        d = u.size // max(n, 1)
        out = np.zeros(d)
        self._weighted_estimate(n, d, int(bool(col_major)), _ptr(u), _ptr(W), _ptr(out))
        return out

    def select_f64(self, idx, state):
        state = np.array(state, dtype=np.float64, order="F", copy=True)
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        N = state.shape[0]
        dim = 1 if state.ndim == 1 else state.shape[1]
        self._select_f64(N, dim, _ptr(idx), _ptr(state))
        return state

    def pf_ar1(self, N, y, phi, sx, sy, sd0, mkey, rkey, scheme=2, threshold=0.5,
               record=True, backend=0):
        y = np.ascontiguousarray(y, dtype=np.float64)
        T = len(y) - 1
        mk = np.array(mkey, dtype=np.uint32)
        rk = np.array(rkey, dtype=np.uint32)
        ll = np.zeros(1)
        ess = np.zeros(T + 1)
        rs = np.zeros(T + 1, dtype=np.uint8)
        anc = np.zeros((T + 1, N), dtype=np.uint64) if record else None
        x = np.zeros(N)
        W = np.zeros(N)
        if self.which == "oracle":
            self._pf_ar1(N, T, _ptr(y), phi, sx, sy, sd0, _ptr(mk), _ptr(rk), scheme, threshold,
                         _ptr(ll), _ptr(ess), _ptr(rs), _ptr(anc), _ptr(x), _ptr(W))
        else:
            self._pf_ar1(N, T, _ptr(y), phi, sx, sy, sd0, _ptr(mk), _ptr(rk), scheme, threshold,
                         backend, _ptr(ll), _ptr(ess), _ptr(rs), _ptr(anc), _ptr(x), _ptr(W),
                         int(record))
        return dict(loglik=float(ll[0]), ess=ess, resampled=rs, anc=anc, x=x, W=W)

    def pf_ar1_digest(self, N, y, phi, sx, sy, sd0, mkey, rkey, scheme=2, threshold=0.5):
        """The reference's BackendSEQ filter with, per resampling iteration t,
        two exact sums of its parent vector: digest[t] = (sum idx_i,
        sum idx_i (i + 1)) (zeros where t did not resample)."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        T = len(y) - 1
        mk = np.array(mkey, dtype=np.uint32)
        rk = np.array(rkey, dtype=np.uint32)
        ll = np.zeros(1)
        ess = np.zeros(T + 1)
        rs = np.zeros(T + 1, dtype=np.uint8)
        dig = np.zeros((T + 1, 2), dtype=np.uint64)
        x = np.zeros(N)
        assert self._pf_ar1_digest(N, T, _ptr(y), phi, sx, sy, sd0, _ptr(mk), _ptr(rk), scheme, threshold,
                                   _ptr(ll), _ptr(ess), _ptr(rs), _ptr(dig), _ptr(x)) == 0
        return dict(loglik=float(ll[0]), ess=ess, resampled=rs, digest=dig, x=x)

    # -- oracle-only helpers ------------------------------------------------
    def simulate_ar1(self, T, phi, sx, sy, sd0, key):
        k = np.array(key, dtype=np.uint32)
        x = np.zeros(T + 1)
        y = np.zeros(T + 1)
        self._simulate_ar1(T, phi, sx, sy, sd0, _ptr(k), _ptr(x), _ptr(y))
        return x, y

    def math_f64(self, fn: str, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        y2 = np.zeros_like(x) if fn == "sincos" else None
        self._math_f64({"log": 0, "exp": 1, "sincos": 2}[fn], len(x), _ptr(x), _ptr(y), _ptr(y2))
        return (y, y2) if fn == "sincos" else y

    def fold(self, x, s0=0.0):
        """Sequential left fold: (prefix values, final value)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        pre = np.zeros_like(x)
        fin = np.zeros(1)
        self._fold(len(x), _ptr(x), s0, _ptr(pre), _ptr(fin))
        return pre, float(fin[0])

    def engine_text(self, eng):
        """The reference's `os << eng` for an engine in state `eng`."""
        buf = ctypes.create_string_buffer(4096)
        e = eng.copy()
        assert self._engine_to_text(ctypes.byref(e), buf, 4096) == 0
        return buf.value.decode()

    def engine_text_roundtrip(self, kind, text):
        """`is >> eng` of `text`, then `os << eng`."""
        buf = ctypes.create_string_buffer(4096)
        e = Engine.make(kind)
        assert self._engine_text_roundtrip(ctypes.byref(e), text.encode(), buf, 4096) == 0
        return buf.value.decode()

    def engine_from_text(self, kind, text):
        """A state read by the reference's `is >> eng`."""
        e = Engine.make(kind)
        assert self._engine_from_text(ctypes.byref(e), text.encode()) == 0
        return e

    def index_matrix(self, idx, iter_back, iter_, col_major):
        """ResampleIndex::read_index_matrix of R pushed vectors idx [R, N];
        returns (matrix [N * R], trace of every id [N])."""
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        R, N = idx.shape
        out = np.zeros(N * (iter_back - iter_ + 1), dtype=np.uint64)
        tr = np.zeros(N, dtype=np.uint64)
        assert self._index_matrix(N, R, _ptr(idx), iter_back, iter_, int(bool(col_major)), _ptr(out), _ptr(tr)) == 0
        return out, tr

    def kalman_ar1(self, y, phi, sx, sy):
        y = np.ascontiguousarray(y, dtype=np.float64)
        ll = np.zeros(1)
        g = np.zeros(3)
        self._kalman_ar1(len(y) - 1, _ptr(y), phi, sx, sy, _ptr(ll), _ptr(g))
        return float(ll[0]), g


def have_ref() -> bool:
    return os.path.exists(REF_SO) and os.path.exists(REF_GENERIC_SO)
