"""Benchmark of the B200 path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mckl_b200|reference]
                    [--workload smc|rng|callers|plain|adjoint] [--filters F] [--obs T] [--parts all|timed]
                    [--sets S] [--particles N]

Workload `smc` (default, the batched SMC configuration): F = 4096 independent
AR(1) bootstrap filters, phi ~ U[0.5, 0.99], sx ~ U[0.5, 2], sy ~ U[0.2, 1] and
particle counts log-uniform in [256, 65536] (47.2 M particles in all), drawn
from Philox4x32(1234); T = 500 observations per filter simulated from the
filter's own seed; systematic resampling when ESS < N/2.  FP32 propagation
and likelihoods, FP64 normaliser, log-likelihood and cumulative scan; one
persistent launch, replayed from a CUDA graph, block shape chosen by the
library's autotuner.  A step is one full pass (every filter, every
observation); `value` is particle-steps per second over all ranks.  Inputs
(parameters, observations) are resident in HBM when timing starts; a step
streams ~1.1 GB of particle state per pass, far above the 126 MB L2, so no
flush is needed.  Also measured in the same run (rank 0):
  * `plain_gpu`: the plain FP64 filter (mckl_b200_pf_ar1_plain_f64, the
    reference's step order) on 32 filters spread over the particle counts,
    one after the other, extrapolated to all F filters by a least-squares
    per-filter cost a + b N; `ratio_vs_plain` = per-GPU value / that rate;
  * `accuracy`: per filter |logL_FP32 - logL_FP64| / |logL_FP64|, with
    logL_FP64 the FP64 shadow run along the same genealogy (same counters,
    same ancestors; target 1e-6), and the estimates' offset from the exact
    Kalman log-likelihood;
  * `adjoint`: the differentiated configuration -- gradients of the FP64
    estimates in (phi, sx, sy) for 256 parameter sets, N = 2^16, T = 1000,
    ancestors fixed, against central finite differences under common random
    numbers and against the Kalman gradient;
  * `rng`: the RNG + distributions configuration (see below), one step.

Workload `rng`: for each of Threefry4x64-20 and ARS-5, seeded 42, 2^28 values
per call: raw u32 words, U01 (the reference's default canonical U01) in fp32
and fp64, Normal(0,1) fp32/fp64, Exponential(1) fp32/fp64, Gamma fp32/fp64
with shape ~ U[0.5, 10] per block of 4096 samples (block b an independent
stream at counter (0, b)), each call from a freshly seeded engine; `value`
is bytes written per second (each output of 1-2 GiB exceeds the L2), plus
the Philox4x32 configuration (2^26 words, then 2^24 U01OO doubles).

With N ranks every rank runs the whole workload on its own keys or counter
range (weak scaling, no data-path collective); time is the max over ranks.

`e2e` is the same step through the public API with host buffers: every step
copies the observations from page-locked host memory into the filters and
reads the F log-likelihoods back (smc); the RNG calls write page-locked host
buffers directly (rng).

`cpu_baseline` and `--impl reference` run the reference's own CPU code (MCKL
compiled from its headers into oracle/_ref) on all host threads, on a bounded
sample of the same workload.

`--parts timed` runs only the warm-up and the timed loop (for profilers);
`--shape 512x2` fixes the batched kernel's block shape instead of autotuning.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batched SMC particle-steps/s vs plain GPU path at matched logL error; RNG GB/s"
LOG2N = 28
# MUFU (special-function unit) results per particle-step in the batched
# kernel: lg2 for the Box-Muller radius, sin|cos for the angle (one pair per
# two particles), ex2 for the weight; nominal 16 results / clock / SM.
MUFU_PER_PS = 3.0
MUFU_PER_CLK_SM = 16
# From the ncu capture summarised in profiles/k_pf_batched_c4.md: warp
# instructions per particle-step of the batched kernel, and DRAM bytes per
# particle-step (read + write), measured on a 2.4e8 particle-step case.
WARP_INSTR_PER_PS = 8.47
DRAM_BYTES_PER_PS = 13.75


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d.get("sm_max_mhz", 1965.0)), "measured"
    return 6650.0, 1965.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def barrier(world):
    if world > 1:
        import torch

        torch.distributed.barrier()


def events():
    import torch

    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


# ---------------------------------------------------------------------------
# SMC workload
# ---------------------------------------------------------------------------
def make_filters(mb, w, **kw):
    return mb.BatchedFilters(w["N"], w["y"], w["phi"], w["sx"], w["sy"], w["mkeys"], w["rkeys"], **kw)


def plain_sample(mb, w, T, nsample=32):
    """Plain FP64 filter on `nsample` filters spread over N; fit t = a + b N."""
    import numpy as np
    import torch

    F = len(w["N"])
    order = np.argsort(w["N"], kind="stable")
    idx = order[np.linspace(0, F - 1, min(nsample, F)).astype(int)]
    ts, ns = [], []
    for f in idx:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        mb.pf_ar1_plain(int(w["N"][f]), w["y"][f], w["phi"][f], w["sx"][f], w["sy"][f], w["sd0"][f],
                        tuple(int(k) for k in w["mkeys"][f]), tuple(int(k) for k in w["rkeys"][f]),
                        scheme=mb.Systematic)
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
        ns.append(float(w["N"][f]))
    A = np.stack([np.ones(len(ns)), np.array(ns)], axis=1)
    coef, *_ = np.linalg.lstsq(A, np.array(ts), rcond=None)
    a, b = max(float(coef[0]), 0.0), max(float(coef[1]), 0.0)
    total = float(np.sum(a + b * w["N"].astype(float)))
    return {"particle_steps_per_s": float(w["N"].sum()) * T / total, "est_seconds_all_filters": total,
            "fit_seconds_per_filter": {"a": a, "b_per_particle": b}, "measured_seconds": float(sum(ts)),
            "sample": f"{len(idx)} filters spread over the particle counts, run one after the other; "
                      "total extrapolated with t_f = a + b N_f (least squares)"}


def bench_smc(args, rank, world, dev):
    import numpy as np
    import torch

    import mckl_b200 as mb

    from mckl_b200.shard import filter_range, job_rate

    T = args.obs
    first, _ = filter_range(rank, args.filters)
    w = mb.batched_workload(F=args.filters, T=T, seed=1234, first=first)
    ps_per_step = float(w["N"].sum()) * T
    b = make_filters(mb, w, threshold=args.threshold)
    if args.shape:
        th, cps = (int(v) for v in args.shape.split("x"))
        b.config(th, cps)
        trials = [(th, cps, 0.0)]
    else:
        trials = b.autotune()
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        b.run(graph=True)
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(dev.index if dev.index is not None else 0)
    clocks.start()
    l0 = mb.launch_count()
    t0, t1 = events()
    t0.record(stream)
    for _ in range(args.steps):
        b.run(graph=True)
    t1.record(stream)
    torch.cuda.synchronize()
    launches = mb.launch_count() - l0
    clk = clocks.stop()
    value, elapsed = job_rate(ps_per_step * args.steps, t0.elapsed_time(t1) / 1e3, world, dev)
    ll, nres = b.results()
    out = dict(value=value, elapsed=elapsed, launches=launches, clocks=clk, ps_per_step=ps_per_step, w=w, ll=ll)
    if args.parts == "timed":
        b.close()
        return out

    # e2e: observations from page-locked host memory every step, results back
    yh = torch.from_numpy(np.ascontiguousarray(w["y"])).pin_memory()
    e2e_steps = max(1, min(args.steps, 3))
    b.set_y(yh)
    b.run(graph=True)
    b.results()
    barrier(world)
    h0, h1 = events()
    h0.record(stream)
    for _ in range(e2e_steps):
        b.set_y(yh)
        b.run(graph=True)
        b.results()
    h1.record(stream)
    torch.cuda.synchronize()
    e2e_value, _ = job_rate(ps_per_step * e2e_steps, h0.elapsed_time(h1) / 1e3, world, dev)
    b.close()
    out["e2e"] = {"value": e2e_value, "unit": "particle-steps/s",
                  "h2d_bytes_per_step": int(w["y"].nbytes), "d2h_bytes_per_step": int(len(w["N"]) * 12)}
    extra = {"autotune": [{"threads": t, "ctas_per_sm": c, "ms": round(m, 3)} for (t, c, m) in trials],
             "resampling_events_per_step": int(nres.sum())}
    if rank == 0:
        from mckl_b200.kalman import kalman_ar1

        bs = make_filters(mb, w, shadow=True, threshold=args.threshold)
        best = min(trials, key=lambda r: r[2])
        bs.config(best[0], best[1])
        bs.run()
        ll32, _ = bs.results()
        ll64 = bs.shadow_loglik()
        bs.close()
        rel = np.abs(ll32 - ll64) / np.abs(ll64)
        kf, _ = kalman_ar1(w["y"], w["phi"], w["sx"], w["sy"])
        extra["accuracy"] = {
            "fp32_vs_fp64_same_genealogy_rel": {"max": float(rel.max()), "median": float(np.median(rel)),
                                                "frac_le_1e-6": float(np.mean(rel <= 1e-6))},
            "estimate_minus_kalman": {"mean": float(np.mean(ll - kf)), "std": float(np.std(ll - kf)),
                                      "max_abs": float(np.max(np.abs(ll - kf)))},
            "target": "|dlogL| <= 1e-6 |logL| against FP64 along the same genealogy"}
        extra["plain_gpu"] = plain_sample(mb, w, T)
        extra["ratio_vs_plain"] = value / world / extra["plain_gpu"]["particle_steps_per_s"]
        extra["ratio_vs_plain_note"] = ("the plain filter run one filter after the other on these filters (each "
                                        "paying its fixed host and launch cost); ratio_vs_plain_c3 divides by the "
                                        "plain path's own rate at N = 2^20 instead")
        # the same batched kernel in FP64 throughout (fp64 handle, its own autotuned shape)
        b64 = make_filters(mb, w, fp64=True, threshold=args.threshold)
        t64 = b64.autotune()
        b64.run(graph=True)
        torch.cuda.synchronize()
        a0, a1 = events()
        reps = 2
        a0.record(stream)
        for _ in range(reps):
            b64.run(graph=True)
        a1.record(stream)
        torch.cuda.synchronize()
        ms64 = a0.elapsed_time(a1) / reps
        ll64, _ = b64.results()
        b64.close()
        best64 = min(t64, key=lambda r: r[2])
        rate64 = ps_per_step / (ms64 / 1e3)
        extra["fp64_batched"] = {
            "particle_steps_per_s": rate64, "ms_per_step": ms64,
            "shape": {"threads": best64[0], "ctas_per_sm": best64[1]},
            "fp32_over_fp64": value / world / rate64,
            "loglik_fp32_minus_fp64_own_genealogy": {"max_abs": float(np.max(np.abs(ll - ll64))),
                                                      "median_abs": float(np.median(np.abs(ll - ll64)))},
            "note": "the batched kernel with FP64 propagation and weights (same counters); each precision "
                    "follows its own genealogy, so the two estimates differ by Monte Carlo noise where an "
                    "ancestor flips; the accuracy bar is taken along one genealogy (accuracy above)"}
    out["extra"] = extra
    return out


def bench_callers(dev, hbm_peak, peak_kind, reps=5):
    """The callers either side of the filters: ResampleIndex's index matrix
    (N = 2^20 particles, R = 100 iterations of parent indices from systematic
    resampling of log-normal weights), SMCEstimator's weighted estimate
    (n = 2^24 particles, d = 4) and the PMCMC caller (64 chains, N = 4096,
    T = 200, 10 iterations).  Device-timed with CUDA events; algorithmic
    bytes: the index matrix reads one parent word per entry and writes one
    (2 x 8 B x N x R), the estimate reads u and W once (8 B x n x (d + 1))."""
    import numpy as np
    import torch

    import mckl_b200 as mb

    out = {}
    stream = torch.cuda.current_stream()
    N, R = 1 << 20, 100
    g = torch.Generator(device="cuda").manual_seed(11)
    rr = mb.Philox4x32(77)
    ri = mb.ResampleIndex()
    for _ in range(R):
        W = torch.exp(torch.randn(N, dtype=torch.float64, device="cuda", generator=g))
        W /= W.sum()
        ri.push_back(N, mb.rep_to_index(mb.resample(mb.Systematic, rr, W), N))
    for name, layout in (("col_major", ri.ColMajor), ("row_major", ri.RowMajor)):
        for _ in range(2):
            ri.index_matrix(layout)
        torch.cuda.synchronize()
        t0, t1 = events()
        t0.record(stream)
        for _ in range(reps):
            ri.index_matrix(layout)
        t1.record(stream)
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / reps
        gbs = 2 * 8 * N * R / ms / 1e6
        out[f"index_matrix_{name}"] = {"ms": round(ms, 4), "GB_s": round(gbs, 1),
                                       "frac_of_hbm": round(gbs / hbm_peak, 3)}
    out["index_matrix_workload"] = f"N = 2^20, R = {R}, one launch + its error-flag read per call"
    del ri
    n, d = 1 << 24, 4
    W = torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
    W /= W.sum()
    for name, col in (("row_major", False), ("col_major", True)):
        u = torch.randn((d, n) if col else (n, d), dtype=torch.float64, device="cuda", generator=g)
        for _ in range(2):
            mb.weighted_estimate(u, W, col_major=col)
        torch.cuda.synchronize()
        t0, t1 = events()
        t0.record(stream)
        for _ in range(reps):
            mb.weighted_estimate(u, W, col_major=col)
        t1.record(stream)
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / reps
        gbs = 8 * n * (d + 1) / ms / 1e6
        out[f"weighted_estimate_{name}"] = {"ms": round(ms, 4), "GB_s": round(gbs, 1),
                                            "frac_of_hbm": round(gbs / hbm_peak, 3)}
        del u
    out["weighted_estimate_workload"] = "n = 2^24, d = 4, FP64; inputs 671 MB, above the 126 MB L2"
    out["hbm_peak"] = {"GB_s": hbm_peak, "kind": peak_kind}
    C, Np, T, iters = 64, 4096, 200, 10
    y = np.concatenate([[0.0], np.cumsum(np.random.default_rng(3).normal(size=T)) * 0.3])
    theta0 = np.tile([0.9, 1.0, 0.5], (C, 1))
    prior = lambda th: 0.0 if (abs(th[0]) < 1 and th[1] > 0 and th[2] > 0) else -np.inf  # noqa: E731
    mb.pmcmc_ar1(y, Np, theta0, [0.02, 0.05, 0.05], prior, 2, seed=5)
    torch.cuda.synchronize()
    t = time.perf_counter()
    mb.pmcmc_ar1(y, Np, theta0, [0.02, 0.05, 0.05], prior, iters, seed=6)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t
    out["pmcmc"] = {"chains": C, "N": Np, "T": T, "iterations": iters, "s": round(dt, 4),
                    "chain_iterations_per_s": round(C * iters / dt, 1),
                    "particle_steps_per_s": C * iters * Np * T / dt,
                    "note": "wall clock (host prior callback and accept step between filter launches)"}
    return out


def bench_plain_c3(N=1 << 20, T=1000):
    """The plain FP64 particle filter (the reference's step order, one
    filter): N = 2^20 particles, T = 1000 observations simulated from
    Philox4x32 key (7, 0) (x_0 ~ N(0, 1 / 0.19), phi = 0.9, sx = 1, sy = 0.5),
    systematic resampling at ESS < N / 2; wall clock with the device
    synchronised (the step loop is host-driven), and the estimate against
    the exact Kalman log-likelihood."""
    import numpy as np
    import torch

    import mckl_b200 as mb
    from mckl_b200.kalman import kalman_ar1

    phi, sx, sy = 0.9, 1.0, 0.5
    sd0 = sx / np.sqrt(1 - phi * phi)
    g = mb.Philox4x32()
    g.key = (7, 0)
    z = mb.normal_distribution(g, 2 * T + 2).cpu().numpy()
    x = sd0 * z[0]
    y = np.zeros(T + 1)
    for t in range(1, T + 1):
        x = phi * x + sx * z[t]
        y[t] = x + sy * z[T + t]
    mb.pf_ar1_plain(N, y[:11], phi, sx, sy, sd0, (11, 0), (12, 0), scheme=mb.Systematic)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = mb.pf_ar1_plain(N, y, phi, sx, sy, sd0, (11, 0), (12, 0), scheme=mb.Systematic)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    kf, _ = kalman_ar1(y, phi, sx, sy)
    # the same filter with resampling off: the weights degenerate (all but a
    # few hundred exactly zero), the hard case for the exact folds
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    res0 = mb.pf_ar1_plain(N, y, phi, sx, sy, sd0, (11, 0), (12, 0), scheme=mb.Systematic, threshold=0.0)
    torch.cuda.synchronize()
    dt0 = time.perf_counter() - t1
    return {"workload": f"plain FP64 particle filter, N = 2^20, T = {T}, systematic resampling at ESS < N/2",
            "particle_steps_per_s": N * T / dt, "s": round(dt, 3), "resampling_steps": int(res["resampled"].sum()),
            "loglik": res["loglik"], "loglik_minus_kalman": float(res["loglik"] - kf[0]),
            "scan_ties": res["ties"],
            "no_resampling": {"particle_steps_per_s": N * T / dt0, "s": round(dt0, 3),
                              "final_ess": float(res0["ess"][-1]),
                              "note": "threshold 0: the weights degenerate, all but a few exactly zero"},
            "scan_ties_note": "uniforms within one representable step of a cumulative weight, over all resampling "
                              "steps; the cumulative weights are the reference's sequential fold bit for bit, so "
                              "a tie flips no ancestor",
            "bound": "latency: per step a chain of ~25 dependent kernels (the exact sequential folds walk their "
                     "windows on one thread) and one host read-back of (ESS, log normaliser), the reference's step "
                     "order; the next step's noise and the next resampling's uniforms run beside it on a second "
                     "stream",
            "y": y}


def cpu_c3_reference(y, N=1 << 20, T=30):
    """The compiled reference's SMCSampler (BackendSEQ, one thread) on the
    same model: N = 2^20 particles, the first T observations."""
    import numpy as np

    import oracle as O

    if not O.have_ref():
        return None
    cpu = O.CPUPath("ref")
    Nv = np.array([N], dtype=np.uint64)
    yy = np.ascontiguousarray(y[:T + 1][None, :])
    phi, sx, sy = (np.array([v]) for v in (0.9, 1.0, 0.5))
    mk = np.array([[11, 0]], dtype=np.uint32)
    rk = np.array([[12, 0]], dtype=np.uint32)
    ll = np.zeros(1)

    def p(a):
        return ctypes.c_void_p(a.ctypes.data)

    t0 = time.perf_counter()
    rc = cpu._pf_ar1_batch(1, p(Nv), T, p(yy), p(phi), p(sx), p(sy), p(mk), p(rk), 2, 0.5, p(ll), 1)
    dt = time.perf_counter() - t0
    if rc != 0:
        return None
    return {"value": N * T / dt, "unit": "particle-steps/s", "cores": 1, "kind": "reference",
            "sample": f"N = 2^20, the first {T} of the 1000 steps; {dt:.1f} s"}


def cpu_callers_reference():
    """The compiled reference's ResampleIndex::read_index_matrix (one thread)
    on N = 2^16, R = 100 (push_back copies included)."""
    import numpy as np

    import oracle as O

    if not O.have_ref():
        return None
    cpu = O.CPUPath("ref")
    N, R = 1 << 16, 100
    idx = np.random.default_rng(1).integers(0, N, size=(R, N)).astype(np.uint64)
    outm = np.zeros(N * R, dtype=np.uint64)
    t = time.perf_counter()
    cpu._index_matrix(N, R, idx.ctypes.data_as(ctypes.c_void_p), R - 1, 0, 1,
                      outm.ctypes.data_as(ctypes.c_void_p), None)
    dt = time.perf_counter() - t
    return {"index_matrix_GB_s": 2 * 8 * N * R / dt / 1e9, "cores": 1, "kind": "reference",
            "sample": "N = 2^16, R = 100 random parents, column-major"}


def bench_adjoint(rank, dev, sets=256, N=1 << 16, T=1000, C=32, threads=1024):
    """Differentiated SMC: gradient of the FP64 estimate in (phi, sx, sy) for
    `sets` parameter sets drawn like the batched workload, N particles, T
    observations, ancestors fixed and replayed from the counters."""
    import numpy as np
    import torch

    import mckl_b200 as mb
    from mckl_b200 import autograd as AG
    from mckl_b200.kalman import kalman_ar1

    w = mb.batched_workload(F=sets, T=T, seed=4321 + 7919 * rank, nmin=N, nmax=N + 1)
    b = mb.BatchedFilters(w["N"], w["y"], w["phi"], w["sx"], w["sy"], w["mkeys"], w["rkeys"], fp64=True)
    b.config(threads, 1)
    b.adjoint(C)  # warm-up (allocates the checkpoint and replay memory)
    stream = torch.cuda.current_stream()
    t0, t1 = events()
    t0.record(stream)
    ll, g = b.adjoint(C)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    b.close()
    w["threads"] = threads
    fd = AG.finite_differences(w, h=1e-5, threads=threads)
    rel_fd = np.abs(g - fd) / np.maximum(np.abs(fd), 1.0)
    # Richardson extrapolation of FD(h) and FD(h/2) removes the h^2 term,
    # separating the differences' truncation error from the adjoint's
    fd2 = AG.finite_differences(w, h=5e-6, threads=threads)
    rich = (4.0 * fd2 - fd) / 3.0
    rel_rich = np.abs(g - rich) / np.maximum(np.abs(rich), 1.0)
    kll, kg = kalman_ar1(w["y"], w["phi"], w["sx"], w["sy"])
    rel_k = np.linalg.norm(g - kg, axis=1) / np.linalg.norm(kg, axis=1)
    cos = np.sum(g * kg, axis=1) / (np.linalg.norm(g, axis=1) * np.linalg.norm(kg, axis=1))
    ps = float(sets) * N * T
    # both estimators over R independent runs (model and resampling keys):
    # the fixed-ancestor adjoint and the consistent score (Fisher identity,
    # PaRIS), each against the Kalman gradient with its Monte Carlo error
    R, score_threads = 8, 512
    b = mb.BatchedFilters(w["N"], w["y"], w["phi"], w["sx"], w["sy"], w["mkeys"], w["rkeys"], fp64=True)
    S = np.zeros((R, sets, 3))
    G = np.zeros((R, sets, 3))
    score_ms = []
    for r in range(R):
        mk, rk = w["mkeys"].copy(), w["rkeys"].copy()
        mk[:, 1] += 1000 * (r + 1)
        rk[:, 1] += 1000 * (r + 1)
        b.set_keys(mk, rk)
        b.config(score_threads, 1)
        e0, e1 = events()
        e0.record(stream)
        _, S[r] = b.score()
        e1.record(stream)
        torch.cuda.synchronize()
        score_ms.append(e0.elapsed_time(e1))
        b.config(threads, 1)
        _, G[r] = b.adjoint(C)
    b.close()

    def vs_kalman(E):
        mean = E.mean(0)
        se = E.std(0, ddof=1) / np.sqrt(R)
        kn = np.linalg.norm(kg, axis=1)
        single = np.linalg.norm(E - kg[None], axis=2) / kn[None]
        return {"rel_norm_of_mean_median": float(np.median(np.linalg.norm(mean - kg, axis=1) / kn)),
                "rel_norm_single_run_median": float(np.median(single)),
                "rel_se_of_mean_median": float(np.median(np.linalg.norm(se, axis=1) / kn)),
                "components_within_3se": float(np.mean(np.abs(mean - kg) <= 3 * se))}

    estimators = {
        "runs": R,
        "adjoint_fixed_ancestors": vs_kalman(G),
        "score_fisher_paris": dict(vs_kalman(S), ms_per_run=float(np.median(score_ms)),
                                   threads=score_threads),
        "definition": "per parameter set: ||mean over runs - Kalman|| / ||Kalman|| (median over sets), the same "
                      "for single runs, the standard error of the mean relative to ||Kalman||, and the fraction "
                      "of components whose mean lies within 3 standard errors of Kalman"}
    return {"workload": f"{sets} parameter sets, N = {N}, T = {T}, FP64, checkpoint every {C} steps, "
                        f"{threads} threads per filter",
            "ms": ms, "forward_particle_steps_per_s": ps / (ms / 1e3),
            "vs_fd_rel": {"max": float(rel_fd.max()), "median": float(np.median(rel_fd)),
                          "frac_le_1e-4": float(np.mean(rel_fd <= 1e-4)),
                          "definition": "|adjoint - central FD (h = 1e-5, common random numbers, base ancestors)| "
                                        "/ max(|FD|, 1)"},
            "vs_richardson_fd_rel": {"max": float(rel_rich.max()), "median": float(np.median(rel_rich)),
                                     "definition": "same, against (4 FD(h/2) - FD(h)) / 3"},
            "vs_kalman": {"rel_norm_median": float(np.median(rel_k)), "cosine_median": float(np.median(cos)),
                          "loglik_minus_kalman_mean": float(np.mean(ll - kll)),
                          "note": "fixed ancestors: a biased estimate of the exact score at any N"},
            "estimators_vs_kalman": estimators}


# ---------------------------------------------------------------------------
# RNG workload
# ---------------------------------------------------------------------------
def rng_ops():
    """(name, engine class name, call, bytes per value)."""
    ops = []
    for eng in ("Threefry4x64", "ARS"):
        ops.append((f"{eng}.rand_u32", eng, "rand", 4))
        ops.append((f"{eng}.u01_f32", eng, "u01_f32", 4))
        ops.append((f"{eng}.u01_f64", eng, "u01_f64", 8))
        ops.append((f"{eng}.normal_f32", eng, "normal_f32", 4))
        ops.append((f"{eng}.normal_f64", eng, "normal_f64", 8))
        ops.append((f"{eng}.exponential_f32", eng, "exp_f32", 4))
        ops.append((f"{eng}.exponential_f64", eng, "exp_f64", 8))
        ops.append((f"{eng}.gamma_f32", eng, "gamma_f32", 4))
        ops.append((f"{eng}.gamma_f64", eng, "gamma_f64", 8))
    return ops


GAMMA_BLOCK = 4096


def gamma_shapes(nvalues):
    """Shape per block of 4096 samples, U[0.5, 10] from the canonical
    uniforms of Philox4x32(43)."""
    import numpy as np

    import mckl_b200 as mb

    nb = nvalues // GAMMA_BLOCK
    g = mb.Philox4x32()
    g.key = (43, 0)
    u = mb.u01_canonical_distribution(g, nb, dtype="f64").cpu().numpy()
    return np.ascontiguousarray(0.5 + 9.5 * u)


def gamma_shapes_cpu(nvalues):
    """The same shapes from the CPU reference path (reference arm only; the
    canonical uniforms are bit-identical)."""
    import numpy as np

    import oracle as O

    nb = nvalues // GAMMA_BLOCK
    u = O.CPUPath("oracle").u01(O.Engine.make(O.PHILOX4X32, key=(43,)), "canonical", True, nb)
    return np.ascontiguousarray(0.5 + 9.5 * u)


def reference_workload(F=4096, T=500, seed=1234, nmin=256, nmax=65536):
    """The batched configuration's parameters and observations made on the
    CPU, for the reference arm (which must not load the library under test):
    the same recipe as mckl_b200.batched_workload -- canonical uniforms of
    Philox4x32(seed) for the parameters and particle counts (bit-identical),
    Normal draws of Philox4x32(f, 10) for filter f's observations (equal to
    the GPU's within 2 ULP)."""
    import numpy as np

    import oracle as O

    orc = O.CPUPath("oracle")
    u = orc.u01(O.Engine.make(O.PHILOX4X32, key=(seed, 0)), "canonical", True, 4 * F).reshape(F, 4)
    phi = 0.5 + 0.49 * u[:, 0]
    sx = 0.5 + 1.5 * u[:, 1]
    sy = 0.2 + 0.8 * u[:, 2]
    N = np.rint(np.exp(np.log(nmin) + (np.log(nmax) - np.log(nmin)) * u[:, 3])).astype(np.uint64)
    z = np.stack([orc.normal(O.Engine.make(O.PHILOX4X32, key=(f, 10)), True, 2 * T + 2) for f in range(F)])
    sd0 = sx / np.sqrt(1 - phi * phi)
    x = sd0 * z[:, 0]
    y = np.zeros((F, T + 1))
    for t in range(1, T + 1):
        x = phi * x + sx * z[:, t]
        y[:, t] = x + sy * z[:, T + t]
    ids = np.arange(F)
    mkeys = np.stack([ids, np.full(F, 11)], axis=1).astype(np.uint32)
    rkeys = np.stack([ids, np.full(F, 12)], axis=1).astype(np.uint32)
    return dict(N=N, y=y, phi=phi, sx=sx, sy=sy, sd0=sd0, mkeys=mkeys, rkeys=rkeys)


def run_op(mb, call, g, n, buf32, buf64):
    import torch

    f32 = buf32.view(torch.float32)
    if call == "rand":
        mb.rand(g, n, buf32)
    elif call == "u01_f32":
        mb.u01_canonical_distribution(g, n, f32)
    elif call == "u01_f64":
        mb.u01_canonical_distribution(g, n, buf64)
    elif call == "normal_f32":
        mb.normal_distribution(g, n, f32)
    elif call == "normal_f64":
        mb.normal_distribution(g, n, buf64)
    elif call == "exp_f32":
        mb.exponential_distribution(g, n, f32)
    elif call == "exp_f64":
        mb.exponential_distribution(g, n, buf64)
    elif call == "gamma_f32":
        mb.gamma_blocks(g, GAMMA_BLOCK, shapes(n), f32)
    elif call == "gamma_f64":
        mb.gamma_blocks(g, GAMMA_BLOCK, shapes(n), buf64)


_SHAPES = {}


def shapes(n):
    if n not in _SHAPES:
        _SHAPES[n] = gamma_shapes(n)
    return _SHAPES[n]


def bench_rng(rank, world, dev, steps, warmup, e2e=True, clocks_on=True):
    import torch

    import mckl_b200 as mb

    n = 1 << LOG2N
    ops = rng_ops()
    buf32 = torch.empty(n, dtype=torch.int32, device=dev)
    buf64 = torch.empty(n, dtype=torch.float64, device=dev)

    from mckl_b200.shard import job_rate, rng_counter

    def fresh(eng):
        g = mb.ENGINES[eng](42)
        g.ctr = rng_counter(rank)  # rank-private counter range
        return g

    stream = torch.cuda.current_stream()

    def step(record=None):
        for (name, eng, call, bpv) in ops:
            if record is not None:
                e0, e1 = events()
                e0.record(stream)
            run_op(mb, call, fresh(eng), n, buf32, buf64)
            if record is not None:
                e1.record(stream)
                record.append((name, e0, e1, n * bpv))

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(dev.index if dev.index is not None else 0) if clocks_on else None
    if clocks:
        clocks.start()
    launches0 = mb.launch_count()
    rec = []
    t0, t1 = events()
    t0.record(stream)
    for _ in range(steps):
        step(rec)
    t1.record(stream)
    torch.cuda.synchronize()
    launches = mb.launch_count() - launches0
    clk = clocks.stop() if clocks else None
    bytes_per_step = sum(n * bpv for (_, _, _, bpv) in ops)
    rate, elapsed = job_rate(bytes_per_step * steps, t0.elapsed_time(t1) / 1e3, world, dev)
    value = rate / 1e9
    per_op = {}
    for (name, e0, e1, nbytes) in rec:
        d = per_op.setdefault(name, {"ms": 0.0, "bytes": nbytes, "calls": 0})
        d["ms"] += e0.elapsed_time(e1)
        d["calls"] += 1
    for d in per_op.values():
        d["ms"] /= d["calls"]
        d["GB_s"] = d["bytes"] / (d["ms"] / 1e3) / 1e9
    # Philox4x32 configuration: 2^26 raw words, then 2^24 U01OO doubles
    p32 = torch.empty(1 << 26, dtype=torch.int32, device=dev)
    p64 = torch.empty(1 << 24, dtype=torch.float64, device=dev)
    for _ in range(3):
        mb.rand(mb.Philox4x32(42), 1 << 26, p32)
    # Kernels of 20-60 us are shorter than a Python call, so each call is
    # captured once in a CUDA graph and the graph replayed: the time is the
    # GPU's, not the interpreter's.
    def graph_ms(fn, reps=50):
        fn()
        torch.cuda.synchronize()
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr):
            fn()
        for _ in range(3):
            gr.replay()
        a, bb = events()
        a.record(stream)
        for _ in range(reps):
            gr.replay()
        bb.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(bb) / reps

    c1 = {}
    for name, fn, nbytes in (("rand_u32_2^26", lambda: mb.rand(mb.Philox4x32(42), 1 << 26, p32), 4 << 26),
                             ("u01oo_f64_2^24", lambda: mb.u01_oo_distribution(mb.Philox4x32(42), 1 << 24, p64),
                              8 << 24),
                             ("store_only_fill_2^26", lambda: p32.fill_(1), 4 << 26)):
        ms = graph_ms(fn)
        c1[name] = {"ms": round(ms, 4), "GB_s": round(nbytes / (ms / 1e3) / 1e9, 1)}
    c1["timing"] = "CUDA graph of one call, replayed 50 times; store_only_fill is torch fill_ on the same 2^26 words"
    out = dict(value=value, elapsed=elapsed, bytes_per_step=bytes_per_step, per_op=per_op, clocks=clk,
               launches=launches, philox_c1=c1)
    if e2e:
        hbuf32 = torch.empty(n, dtype=torch.int32, pin_memory=True)
        hbuf64 = torch.empty(n, dtype=torch.float64, pin_memory=True)
        torch.cuda.synchronize()
        barrier(world)
        h0, h1 = events()
        h0.record(stream)
        for (name, eng, call, bpv) in ops:
            run_op(mb, call, fresh(eng), n, hbuf32, hbuf64)
        h1.record(stream)
        torch.cuda.synchronize()
        e2e_rate, _ = job_rate(bytes_per_step, h0.elapsed_time(h1) / 1e3, world, dev)
        out["e2e"] = {"value": e2e_rate / 1e9, "unit": "GB/s",
                      "h2d_bytes_per_step": 0, "d2h_bytes_per_step": bytes_per_step,
                      "note": "kernels write page-locked host buffers directly"}
    return out


# ---------------------------------------------------------------------------
# CPU: the reference's own code (oracle/_ref) on all host threads
# ---------------------------------------------------------------------------
def cpu_smc_reference(w, T, nfilters=64):
    """One BackendSEQ SMCSampler per filter, OpenMP over a sample of filters."""
    import numpy as np

    import oracle as O

    if not O.have_ref():
        return None
    cpu = O.CPUPath("ref")
    threads = int(cpu._max_threads())
    F = len(w["N"])
    order = np.argsort(w["N"], kind="stable")
    idx = order[np.linspace(0, F - 1, min(nfilters, F)).astype(int)]
    N = np.ascontiguousarray(w["N"][idx], dtype=np.uint64)
    y = np.ascontiguousarray(w["y"][idx])
    phi, sx, sy = (np.ascontiguousarray(w[k][idx]) for k in ("phi", "sx", "sy"))
    mk = np.ascontiguousarray(w["mkeys"][idx], dtype=np.uint32)
    rk = np.ascontiguousarray(w["rkeys"][idx], dtype=np.uint32)
    ll = np.zeros(len(idx))

    def p(a):
        return ctypes.c_void_p(a.ctypes.data)

    t0 = time.perf_counter()
    rc = cpu._pf_ar1_batch(len(idx), p(N), T, p(y), p(phi), p(sx), p(sy), p(mk), p(rk), 2, 0.5, p(ll), threads)
    dt = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError("reference particle filter failed")
    return dict(value=float(N.sum()) * T / dt, unit="particle-steps/s", cores=threads, kind="reference", seconds=dt,
                sample=f"{len(idx)} of the {F} filters spread over the particle counts ({int(N.sum())} particles, "
                       f"T = {T}): MCKL SMCSampler + BackendSEQ per filter, OpenMP over filters; {dt:.1f} s")


def cpu_rng_reference(sample_log2=24):
    import numpy as np

    import oracle as O

    if not O.have_ref():
        return None
    cpu = O.CPUPath("ref")
    threads = int(cpu._max_threads())
    n = 1 << sample_log2
    out = np.empty(n * 2, dtype=np.float64)
    total_bytes, total_s = 0, 0.0
    for (name, eng, call, bpv) in rng_ops():
        e = O.Engine.make(3 if eng == "Threefry4x64" else 5, key=(42,))
        if call.startswith("gamma"):
            a = gamma_shapes_cpu(n)
            t0 = time.perf_counter()
            rc = cpu._gamma_blocks(ctypes.byref(e), int(call.endswith("f64")), len(a), GAMMA_BLOCK,
                                   ctypes.c_void_p(a.ctypes.data), 1.0, ctypes.c_void_p(out.ctypes.data), threads)
            s = time.perf_counter() - t0
            if rc != 0:
                raise RuntimeError("reference gamma failed")
        elif call == "rand":
            s = cpu._fill_u32_parallel(ctypes.byref(e), n, ctypes.c_void_p(out.ctypes.data), threads)
        else:
            dist = {"u01": 0, "normal": 5, "exp": 6}[call.split("_")[0]]
            s = cpu._dist_parallel(ctypes.byref(e), dist, int(call.endswith("f64")), n,
                                   ctypes.c_void_p(out.ctypes.data), threads)
        total_bytes += n * bpv
        total_s += s
    return dict(value=total_bytes / total_s / 1e9, unit="GB/s", cores=threads, kind="reference", seconds=total_s,
                sample=f"every call of the workload at 2^{sample_log2} values (1/{1 << (LOG2N - sample_log2)} "
                       f"of the full size), OpenMP over block-aligned counter ranges")


def strip(d):
    return {k: v for k, v in d.items() if k in ("value", "unit", "cores", "kind", "sample")}


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mckl_b200", choices=["mckl_b200", "reference"])
    ap.add_argument("--workload", default="smc", choices=["smc", "rng", "callers", "plain", "adjoint"],
                    help="callers: only the index matrix / weighted estimate / PMCMC measurements; plain: only the "
                         "plain FP64 filter at N = 2^20 (T = --obs, 1000 by default); adjoint: only the "
                         "differentiated configuration (--sets parameter sets x --particles x T = --obs, 1000 by "
                         "default); one JSON object each")
    ap.add_argument("--sets", type=int, default=256, help="parameter sets of the adjoint workload")
    ap.add_argument("--particles", type=int, default=1 << 16, help="particles per set of the adjoint workload")
    ap.add_argument("--filters", type=int, default=4096)
    ap.add_argument("--obs", type=int, default=500)
    ap.add_argument("--parts", default="all", choices=["all", "timed"])
    ap.add_argument("--threshold", type=float, default=0.5,
                    help="resample when ESS < threshold N (0: never, above 1: every step)")
    ap.add_argument("--shape", default="", help="threads x CTAs per SM (e.g. 512x2) instead of the autotuner")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    smc = args.workload == "smc"
    if smc:
        cfg = {"workload": f"batched SMC: {args.filters} AR(1) bootstrap filters, N log-uniform in [256, 65536], "
                           f"T = {args.obs}, systematic resampling at ESS < {args.threshold:g} N, FP32 propagation + FP64 "
                           "normaliser/scan/logL, one persistent launch replayed from a CUDA graph",
               "filters": args.filters, "T": args.obs,
               "parallelism": f"{world} rank(s), {args.filters} filters each (own seeds)",
               "l2_flush": "none: one step streams ~1.1 GB of particle state, far above the 126 MB L2"}
    else:
        cfg = {"workload": "rng: Threefry4x64-20 and ARS-5 (seed 42), 2^28 values per call: raw u32, U01 "
                           "(canonical) f32/f64, Normal(0,1) f32/f64, Exponential(1) f32/f64, Gamma f32/f64 with shape "
                           "U[0.5, 10] per block of 4096 (block b: counter (0, b))",
               "values_per_call": 1 << LOG2N,
               "l2_flush": "none needed: every output (1-2 GiB) exceeds the 126 MB L2",
               "parallelism": f"{world} independent rank(s), counter range per rank"}

    if args.impl == "reference":
        if rank != 0:
            return
        if args.workload == "callers":
            print(json.dumps({"impl": "reference", "workload": "callers", "cpu_reference": cpu_callers_reference()}))
            return
        if smc:
            w = reference_workload(F=args.filters, T=args.obs, seed=1234)
        vals, secs, base = [], [], None
        for i in range(args.warmup + args.steps):
            r = cpu_smc_reference(w, args.obs, 128) if smc else cpu_rng_reference()
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built on this host"}))
                return
            if i >= args.warmup:
                vals.append(r["value"])
                secs.append(r["seconds"])
                base = r
        v = statistics.median(vals)
        unit = "particle-steps/s" if smc else "GB/s"
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.median(secs) * 1e3,
                "step": "one bounded sample of the workload on the host cores (cpu_baseline.sample)",
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if smc else "u32/f32/f64", "data": "synthetic",
                "config": cfg, "cpu_baseline": strip(dict(base, value=v)),
                "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch

    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    hbm_peak, sm_max, peak_kind = measured_peaks()
    if args.workload == "plain":
        if rank == 0:
            T = args.obs if args.obs != 500 else 1000
            c3 = bench_plain_c3(T=T)
            c3.pop("y")
            print(json.dumps({"workload": "plain", "n_gpus": 1, "plain_c3": c3}))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload == "adjoint":
        if rank == 0:
            T = args.obs if args.obs != 500 else 1000
            adj = bench_adjoint(rank, dev, sets=args.sets, N=args.particles, T=T)
            print(json.dumps({"workload": "adjoint", "n_gpus": 1, "adjoint": adj}))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload == "callers":
        if rank == 0:
            out = {"workload": "callers", "n_gpus": 1, "callers": bench_callers(dev, hbm_peak, peak_kind)}
            cc = cpu_callers_reference()
            if cc:
                out["callers"]["cpu_reference"] = cc
            print(json.dumps(out))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if smc:
        res = bench_smc(args, rank, world, dev)
        sm_mhz = (res["clocks"] or {}).get("sm_mhz") or sm_max
        achieved = res["value"] / world * MUFU_PER_PS / 1e9
        peak = 148 * MUFU_PER_CLK_SM * sm_max / 1e3
        line = {
            "metric": METRIC, "value": res["value"], "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["elapsed"] / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic: AR(1) observations simulated from per-filter Philox4x32 seeds", "config": cfg,
            "roofline": {"bound": "mufu", "kernel": "k_pf_batched<float>", "achieved": achieved, "peak": peak,
                         "unit": "Gop/s", "frac": achieved / peak,
                         "traffic": DRAM_BYTES_PER_PS * res["ps_per_step"],
                         "traffic_note": "DRAM bytes per launch: ncu bytes per particle-step on a medium case x "
                                         "particle-steps per launch (profiles/k_pf_batched_c4.md)",
                         "issue_slots": {"achieved": res["value"] / world * WARP_INSTR_PER_PS / 1e9,
                                         "peak": 148 * 4 * sm_max / 1e3, "unit": "G warp-instr/s",
                                         "frac": res["value"] / world * WARP_INSTR_PER_PS / (148 * 4 * sm_max * 1e6),
                                         "note": "the binding resource: ncu warp-instructions per particle-step x "
                                                 "particle-steps/s against one issue per clock per SM sub-partition"},
                         "peak_kind": "nominal: 16 MUFU results/clk/SM x 148 SMs x clocks.max.sm (the measured "
                                      "peaks file has no MUFU figure)",
                         "at_sampled_clock_frac": achieved / (148 * MUFU_PER_CLK_SM * sm_mhz / 1e3),
                         "note": f"{MUFU_PER_PS:g} MUFU results per particle-step"},
            "e2e": res.get("e2e"), "gpu_launches": res["launches"], "clocks": res["clocks"],
        }
        line.update(res.get("extra", {}))
        if args.parts == "all":
            if rank == 0:
                line["adjoint"] = bench_adjoint(rank, dev)
            rng = bench_rng(rank, world, dev, steps=1, warmup=1, e2e=False, clocks_on=False)
            ph = rng["philox_c1"]["rand_u32_2^26"]["GB_s"]
            line["rng"] = {"value_GB_s": rng["value"],
                           "per_op": {k: {"ms": round(v["ms"], 4), "GB_s": round(v["GB_s"], 1)}
                                      for k, v in rng["per_op"].items()},
                           "philox4x32_config": rng["philox_c1"],
                           "roofline": {"bound": "hbm", "kernel": "k_blocks<PhiloxGen> (2^26 raw words)",
                                        "achieved": ph, "peak": hbm_peak, "unit": "GB/s",
                                        "peak_kind": f"{peak_kind} hbm_gbs", "frac": ph / hbm_peak,
                                        "frac_of_store_only_fill":
                                            ph / rng["philox_c1"]["store_only_fill_2^26"]["GB_s"]}}
            if rank == 0:
                line["callers"] = bench_callers(dev, hbm_peak, peak_kind)
                c3 = bench_plain_c3()
                y3 = c3.pop("y")
                if world == 1:
                    c3["cpu_reference"] = cpu_c3_reference(y3)
                line["plain_c3"] = c3
                if "particle_steps_per_s" in c3 and c3["particle_steps_per_s"] > 0:
                    line["ratio_vs_plain_c3"] = res["value"] / world / c3["particle_steps_per_s"]
            if rank == 0 and world == 1:
                cc = cpu_callers_reference()
                if cc:
                    line["callers"]["cpu_reference"] = cc
                cb = cpu_smc_reference(res["w"], args.obs, 128)
                if cb:
                    line["cpu_baseline"] = strip(cb)
    else:
        res = bench_rng(rank, world, dev, steps=args.steps, warmup=args.warmup)
        dom_name = max(res["per_op"], key=lambda k: res["per_op"][k]["ms"])
        dom = res["per_op"][dom_name]
        line = {
            "metric": METRIC, "value": res["value"], "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["elapsed"] / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32/f32/f64",
            "data": "synthetic: counter-based streams, no input data", "config": cfg,
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": dom["GB_s"], "peak": hbm_peak,
                         "peak_kind": f"{peak_kind} hbm_gbs", "unit": "GB/s", "frac": dom["GB_s"] / hbm_peak,
                         "traffic": None},
            "e2e": res["e2e"], "gpu_launches": res["launches"], "clocks": res["clocks"],
            "per_op": {k: {"ms": round(v["ms"], 4), "GB_s": round(v["GB_s"], 1)} for k, v in res["per_op"].items()},
            "philox4x32_config": res["philox_c1"],
        }
        if rank == 0 and world == 1:
            cb = cpu_rng_reference()
            if cb:
                line["cpu_baseline"] = cb
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
