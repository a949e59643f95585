"""Benchmark of the B200 path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mckl_b200|reference]
                    [--workload rng]

Workload `rng` (the RNG + distributions configuration): for each of
Threefry4x64-20 and ARS-5, seeded 42, streams of 2^28 values as
  raw u32 words, U01 (the reference's default U01Distribution = canonical) in
  fp32 and fp64, Normal(0,1) in fp32 and fp64, Exponential(1) in fp32 and fp64.
Every transform starts from a freshly seeded engine, exactly like one call of
the reference's batch API.  `value` is the bytes written per second over the
whole step (all ranks); outputs (1-2 GiB per call) are far larger than the
126 MB L2, so no flush is needed between calls.  With N ranks each rank runs
the same workload on its own counter range (ctr[1] = rank): weak scaling, no
data-path collective.

`e2e` times the same calls through the same C ABI with page-locked HOST output
buffers (the kernels write the words straight over the host link, as a drop-in
for the reference's host-memory `rand(rng, n, r)` calls).

`cpu_baseline` / `--impl reference` time the reference's own CPU code (MCKL
compiled from its headers into oracle/_ref) with all host threads on a bounded
sample of the same calls.
"""
from __future__ import annotations

import argparse
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


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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
    return ops


def run_op(mb, call, g, n, buf32, buf64):
    if call == "rand":
        mb.rand(g, n, buf32)
    elif call == "u01_f32":
        mb.u01_canonical_distribution(g, n, _as_f32(buf32))
    elif call == "u01_f64":
        mb.u01_canonical_distribution(g, n, buf64)
    elif call == "normal_f32":
        mb.normal_distribution(g, n, _as_f32(buf32))
    elif call == "normal_f64":
        mb.normal_distribution(g, n, buf64)
    elif call == "exp_f32":
        mb.exponential_distribution(g, n, _as_f32(buf32))
    elif call == "exp_f64":
        mb.exponential_distribution(g, n, buf64)


def _as_f32(t):
    import torch

    return t.view(torch.float32)


def bench_rng(args, rank, world, dev):
    import torch

    import mckl_b200 as mb

    n = 1 << LOG2N
    ops = rng_ops()
    buf32 = torch.empty(n, dtype=torch.int32, device=dev)
    buf64 = torch.empty(n, dtype=torch.float64, device=dev)

    def fresh(eng):
        g = mb.ENGINES[eng](42)
        g.ctr = (0, rank)  # rank-private counter range
        return g

    stream = torch.cuda.current_stream()

    def step(record=None):
        for (name, eng, call, bpv) in ops:
            if record is not None:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            run_op(mb, call, fresh(eng), n, buf32, buf64)
            if record is not None:
                e1.record(stream)
                record.append((name, e0, e1, n * bpv))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(dev.index if dev.index is not None else 0)
    clocks.start()
    launches0 = mb.launch_count()
    rec = []
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        step(rec)
    t1.record(stream)
    torch.cuda.synchronize()
    launches = mb.launch_count() - launches0
    clk = clocks.stop()
    elapsed = t0.elapsed_time(t1) / 1e3
    if world > 1:
        t = torch.tensor([elapsed], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        elapsed = float(t.item())
        torch.distributed.barrier()
    bytes_per_step = sum(n * bpv for (_, _, _, bpv) in ops)
    value = world * bytes_per_step * args.steps / elapsed / 1e9
    per_op = {}
    for (name, e0, e1, nbytes) in rec:
        ms = e0.elapsed_time(e1)
        d = per_op.setdefault(name, {"ms": 0.0, "bytes": nbytes, "calls": 0})
        d["ms"] += ms
        d["calls"] += 1
    for d in per_op.values():
        d["ms"] /= d["calls"]
        d["GB_s"] = d["bytes"] / (d["ms"] / 1e3) / 1e9
    dominant = max(per_op, key=lambda k: per_op[k]["ms"])

    # e2e: same calls, page-locked host outputs written by the kernels directly
    hbuf32 = torch.empty(n, dtype=torch.int32, pin_memory=True)
    hbuf64 = torch.empty(n, dtype=torch.float64, pin_memory=True)
    e2e_steps = max(1, min(2, args.steps))
    for (name, eng, call, bpv) in ops[:1]:
        run_op(mb, call, fresh(eng), n, hbuf32, hbuf64)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    h0 = torch.cuda.Event(enable_timing=True)
    h1 = torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(e2e_steps):
        for (name, eng, call, bpv) in ops:
            run_op(mb, call, fresh(eng), n, hbuf32, hbuf64)
    h1.record(stream)
    torch.cuda.synchronize()
    e2e_elapsed = h0.elapsed_time(h1) / 1e3
    if world > 1:
        t = torch.tensor([e2e_elapsed], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_elapsed = float(t.item())
    e2e_value = world * bytes_per_step * e2e_steps / e2e_elapsed / 1e9
    # Philox4x32 configuration: 2^26 raw words, then 2^24 U01OO doubles from the same stream
    g = mb.Philox4x32(42)
    p32 = torch.empty(1 << 26, dtype=torch.int32, device=dev)
    p64 = torch.empty(1 << 24, dtype=torch.float64, device=dev)
    for _ in range(3):
        mb.rand(mb.Philox4x32(42), 1 << 26, p32)
    c1 = {}
    for name, fn, nbytes in (("rand_u32_2^26", lambda gg: mb.rand(gg, 1 << 26, p32), 4 << 26),
                             ("u01oo_f64_2^24", lambda gg: mb.u01_oo_distribution(gg, 1 << 24, p64), 8 << 24)):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        reps = 50
        a.record(stream)
        for _ in range(reps):
            fn(mb.Philox4x32(42))
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / reps
        c1[name] = {"ms": round(ms, 4), "GB_s": round(nbytes / (ms / 1e3) / 1e9, 1)}
    return dict(value=value, elapsed=elapsed, bytes_per_step=bytes_per_step, per_op=per_op, dominant=dominant,
                philox_c1=c1,
                clocks=clk, launches=launches, e2e=dict(value=e2e_value, unit="GB/s", h2d_bytes_per_step=0,
                                                        d2h_bytes_per_step=bytes_per_step,
                                                        note="kernels write page-locked host buffers directly"))


def cpu_rng_baseline(sample_log2=24, reps=1):
    """The reference's CPU fills (oracle/_ref) on all host threads."""
    import ctypes

    import numpy as np

    import oracle as O

    if O.have_ref():
        cpu = O.CPUPath("ref")
        kind = "reference"
        threads = int(cpu._max_threads())
    else:
        return None
    n = 1 << sample_log2
    out = np.empty(n * 2, dtype=np.float64)
    total_bytes, total_s = 0, 0.0
    for _ in range(reps):
        for (name, eng, call, bpv) in rng_ops():
            e = O.Engine.make(3 if eng == "Threefry4x64" else 5, key=(42,))
            if call == "rand":
                s = cpu._fill_u32_parallel(ctypes.byref(e), n, ctypes.c_void_p(out.ctypes.data), threads)
            else:
                dist = {"u01": 0, "normal": 5, "exp": 6}[call.split("_")[0]]
                s = cpu._dist_parallel(ctypes.byref(e), dist, int(call.endswith("f64")), n,
                                       ctypes.c_void_p(out.ctypes.data), threads)
            total_bytes += n * bpv
            total_s += s
    return dict(value=total_bytes / total_s / 1e9, unit="GB/s", cores=threads, kind=kind,
                sample=f"every call of the workload at 2^{sample_log2} values (1/{1 << (LOG2N - sample_log2)} "
                       f"of the full size), OpenMP over block-aligned counter ranges")


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mckl_b200", choices=["mckl_b200", "reference"])
    ap.add_argument("--workload", default="rng", choices=["rng"])
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = {"workload": "rng: Threefry4x64-20 and ARS-5 (seed 42), 2^28 values per call: raw u32, U01 "
                       "(canonical) f32/f64, Normal(0,1) f32/f64, Exponential(1) f32/f64",
           "values_per_call": 1 << LOG2N, "l2_flush": "none needed: every output (1-2 GiB) exceeds the 126 MB L2",
           "parallelism": f"{world} independent rank(s), counter range per rank"}

    if args.impl == "reference":
        if rank != 0:
            return
        steps = []
        for i in range(args.warmup + args.steps):
            r = cpu_rng_baseline(sample_log2=24)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built on this host"}))
                return
            if i >= args.warmup:
                steps.append(r)
        v = statistics.median(s["value"] for s in steps)
        base = steps[0]
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u32/f32/f64", "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": v, "unit": "GB/s", "cores": base["cores"], "kind": base["kind"],
                                 "sample": base["sample"]},
                "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch

    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    res = bench_rng(args, rank, world, dev)
    peak, peak_kind = measured_peaks()
    dom = res["per_op"][res["dominant"]]
    line = {
        "metric": METRIC, "value": res["value"], "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res["elapsed"] / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32/f32/f64",
        "data": "synthetic: counter-based streams, no input data", "config": cfg,
        "roofline": {"bound": "hbm", "kernel": res["dominant"], "achieved": dom["GB_s"], "peak": peak,
                     "peak_kind": f"{peak_kind} hbm_gbs", "unit": "GB/s", "frac": dom["GB_s"] / peak,
                     "traffic": None},
        "e2e": res["e2e"], "gpu_launches": res["launches"], "clocks": res["clocks"],
        "per_op": {k: {"ms": round(v["ms"], 4), "GB_s": round(v["GB_s"], 1)} for k, v in res["per_op"].items()},
        "philox4x32_config": res["philox_c1"],
    }
    if rank == 0 and world == 1:
        cb = cpu_rng_baseline(sample_log2=24)
        line["cpu_baseline"] = cb
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
