"""Generate the golden fixtures in this directory from the reference itself.

Runs the MCKL reference compiled from its own headers (oracle/_ref, built by
``make -C oracle ref``) and writes ``golden.npz``: engine streams and states,
U01 / Normal / Exponential / Gamma samples, Weight normalisation, the six
resampling schemes with their parent indices, and a short particle-filter run
with every ancestor vector.  Before writing, the seed-1 streams are checked
against the reference's own known-answer files
(example/random/random_<engine>[_64].data).

    python tests/golden/make_golden.py          # golden.npz
    python tests/golden/make_golden.py --c3     # c3_full.npz (plain filter, N = 2^20, T = 1000)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

KAT_FILES = {1: "philox4x32", 2: "philox4x32_64", 3: "threefry4x64", 4: "threefry4x64_64", 5: "ars", 6: "ars_64"}


def state_arr(e):
    return np.array(list(e.ctr) + list(e.key) + list(e.tweak) + [e.index, e.kind], dtype=np.uint64)


def main():
    O.build(ref=True)
    ref = O.CPUPath("ref")
    ref_generic = O.CPUPath("ref_generic")
    g = {}
    for kind, name in KAT_FILES.items():
        for seed in (1, 42):
            e = O.Engine.make(kind, key=(seed,))
            words = ref.rand(e, 1000)
            if seed == 1:
                kat = np.loadtxt(os.path.join(O.REF_ROOT, "example", "random", f"random_{name}.data"), dtype=np.uint64)
                assert np.array_equal(words.astype(np.uint64), kat), name
            g[f"rand_{kind}_{seed}"] = words
            g[f"rand_{kind}_{seed}_state"] = state_arr(e)
        # a start in the middle of a block, a counter near the 64-bit carry and
        # a key with two nonzero words (ARS: the reference's generic path)
        e = O.Engine.make(kind, key=(42, 7), ctr=(2**64 - 3, 5), index=1)
        g[f"rand_{kind}_carry"] = (ref_generic if kind in (5, 6) else ref).rand(e, 777)
        g[f"rand_{kind}_carry_state"] = state_arr(e)
    for kind in (1, 3, 5, 2):
        for var in O.U01_VARIANTS:
            for f64 in (False, True):
                e = O.Engine.make(kind, key=(42,), ctr=(3,), index=1)
                g[f"u01_{kind}_{var}_{int(f64)}"] = ref.u01(e, var, f64, 1501)
                g[f"u01_{kind}_{var}_{int(f64)}_state"] = state_arr(e)
        for f64 in (False, True):
            for (mean, sd) in ((0.0, 1.0), (1.5, 2.0)):
                e = O.Engine.make(kind, key=(42,))
                g[f"normal_{kind}_{int(f64)}_{mean}"] = ref.normal(e, f64, 4097, mean, sd)
                g[f"normal_{kind}_{int(f64)}_{mean}_state"] = state_arr(e)
            e = O.Engine.make(kind, key=(42,))
            g[f"exp_{kind}_{int(f64)}"] = ref.exponential(e, f64, 5000, 2.0)
            g[f"exp_{kind}_{int(f64)}_state"] = state_arr(e)
            for alpha in (0.3, 0.7, 1.0, 2.5, 9.7):
                e = O.Engine.make(kind, key=(42,))
                g[f"gamma_{kind}_{int(f64)}_{alpha}"] = ref.gamma(e, f64, 4096, alpha, 1.0)
                g[f"gamma_{kind}_{int(f64)}_{alpha}_state"] = state_arr(e)
    rng = np.random.default_rng(20240601)
    v = rng.normal(size=5000) * 4
    W, ess = ref.weight_set_log(v)
    g["weight_v"], g["weight_W"], g["weight_ess"] = v, W, np.array([ess])
    v2 = rng.normal(size=5000) * 2
    W2, ess2 = ref.weight_add_log(W, v2)
    g["weight_v2"], g["weight_W2"], g["weight_ess2"] = v2, W2, np.array([ess2])
    for scheme in range(6):
        for M in (5000, 3333, 7777):
            e = O.Engine.make(1, key=(9,))
            rep = ref.resample(scheme, e, W2, M)
            g[f"rs_{scheme}_{M}_rep"] = rep
            g[f"rs_{scheme}_{M}_idx"] = ref.rep_index(rep, M)
            g[f"rs_{scheme}_{M}_state"] = state_arr(e)
    orc = O.CPUPath("oracle")
    sd0 = 1 / np.sqrt(1 - 0.9 * 0.9)
    x, y = orc.simulate_ar1(40, 0.9, 1.0, 0.5, sd0, (7, 0))
    g["pf_y"] = y
    for scheme in (0, 1, 2, 3):
        res = ref.pf_ar1(2000, y, 0.9, 1.0, 0.5, sd0, (11, 0), (12, 0), scheme)
        g[f"pf_{scheme}_loglik"] = np.array([res["loglik"]])
        g[f"pf_{scheme}_anc"] = res["anc"][res["resampled"] == 1].astype(np.uint16)
        g[f"pf_{scheme}_resampled"] = res["resampled"]
        g[f"pf_{scheme}_ess"] = res["ess"]
        g[f"pf_{scheme}_x"] = res["x"]
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **g)
    print("wrote", os.path.join(HERE, "golden.npz"), len(g), "arrays")


C3_N, C3_T = 1 << 20, 1000


def _c3_scheme(scheme):
    """One scheme of the plain-filter configuration through the reference's
    SMCSampler + BackendSEQ (a worker of make_c3)."""
    ref = O.CPUPath("ref")
    orc = O.CPUPath("oracle")
    sd0 = 1 / np.sqrt(1 - 0.9 * 0.9)
    _, y = orc.simulate_ar1(C3_T, 0.9, 1.0, 0.5, sd0, (7, 0))
    res = ref.pf_ar1_digest(C3_N, y, 0.9, 1.0, 0.5, sd0, (11, 0), (12, 0), scheme)
    x = res["x"]
    return scheme, y, res["resampled"], res["digest"], res["loglik"], res["ess"], \
        np.array([x.sum(), x.min(), x.max()])


def make_c3():
    """``c3_full.npz``: the plain-filter configuration (AR(1), phi 0.9, sx 1,
    sy 0.5, T = 1000 observations simulated from seed 7, N = 2^20, model key
    (11, 0), resampling key (12, 0), threshold 0.5) for the multinomial,
    stratified, systematic and residual schemes: every iteration's resampling
    decision, two exact sums of every parent vector (sum idx_i and
    sum idx_i (i + 1)), the ESS history, the log-likelihood and the final
    particles' sum / min / max.  About a minute per scheme on one core; the
    four schemes run in parallel processes."""
    import multiprocessing as mp

    O.build(ref=True)
    with mp.get_context("spawn").Pool(4) as pool:
        out = pool.map(_c3_scheme, [0, 1, 2, 3])
    g = {"y": out[0][1], "N": np.array([C3_N])}
    for scheme, _, rs, dig, ll, ess, xs in out:
        g[f"s{scheme}_resampled"] = rs
        g[f"s{scheme}_digest"] = dig
        g[f"s{scheme}_loglik"] = np.array([ll])
        g[f"s{scheme}_ess"] = ess
        g[f"s{scheme}_x"] = xs
    np.savez_compressed(os.path.join(HERE, "c3_full.npz"), **g)
    print("wrote", os.path.join(HERE, "c3_full.npz"), len(g), "arrays")


if __name__ == "__main__":
    if "--c3" in sys.argv:
        make_c3()
    else:
        main()
