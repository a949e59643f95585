"""The N > 1 path of the batched workloads on CPU: two gloo ranks, as one
process per GPU would run them.  The ranks' filter ranges and RNG counter
ranges are disjoint and cover the global workload, and the whole-job rate is
the units summed over ranks over the slowest rank's time, with every rank
taking the same collective steps.  Each rank also runs real work on its shard
-- the oracle's particle filter on its filters of a batched workload and a
fill of its counter range -- and the gathered results must equal a single
process running the whole workload."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from mckl_b200 import shard  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, F, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first, last = shard.filter_range(rank, F)
        units = float(sum(range(first, last)) + 1)  # uneven work per rank
        seconds = 0.5 + rank  # the slower rank sets the time
        rate, t = shard.job_rate(units, seconds, world)
        rate2, t2 = shard.job_rate(2 * units, seconds, world)  # the same steps again
        q.put((rank, first, last, shard.rng_counter(rank), units, rate, t, rate2, t2))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_rate():
    world, F = 2, 4096
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, F, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ranges = [(r[1], r[2]) for r in res]
    assert ranges == [(0, F), (F, 2 * F)]  # disjoint, covering [0, 2F)
    assert len({r[3] for r in res}) == world  # distinct counter ranges
    total = sum(r[4] for r in res)
    tmax = max(0.5 + r[0] for r in res)
    for r in res:
        assert r[6] == tmax and r[5] == pytest.approx(total / tmax)
        assert r[8] == tmax and r[7] == pytest.approx(2 * total / tmax)


def test_single_rank_needs_no_collective():
    assert shard.job_rate(10.0, 2.0, 1) == (5.0, 2.0)
    assert shard.filter_range(0, 7) == (0, 7)


def cpu_workload(F, T, seed, first, nmin=256, nmax=1024):
    """Filters first .. first + F - 1 of the batched workload recipe
    (mckl_b200.batched_workload), made with the oracle on the CPU: parameters
    and particle counts from the canonical uniforms of Philox4x32(seed), four
    per filter in filter order, observations of filter f from the Normal
    draws of Philox4x32(f, 10)."""
    orc = O.CPUPath("oracle")
    u = orc.u01(O.Engine.make(O.PHILOX4X32, key=(seed, 0)), "canonical", True, 4 * (first + F))
    u = u.reshape(first + F, 4)[first:]
    phi = 0.5 + 0.49 * u[:, 0]
    sx = 0.5 + 1.5 * u[:, 1]
    sy = 0.2 + 0.8 * u[:, 2]
    N = np.rint(np.exp(np.log(nmin) + (np.log(nmax) - np.log(nmin)) * u[:, 3])).astype(np.uint64)
    sd0 = sx / np.sqrt(1 - phi * phi)
    y = np.zeros((F, T + 1))
    for k in range(F):
        z = orc.normal(O.Engine.make(O.PHILOX4X32, key=(first + k, 10)), True, 2 * T + 2)
        x = sd0[k] * z[0]
        for t in range(1, T + 1):
            x = phi[k] * x + sx[k] * z[t]
            y[k, t] = x + sy[k] * z[T + t]
    ids = np.arange(first, first + F)
    return dict(N=N, y=y, phi=phi, sx=sx, sy=sy, sd0=sd0, ids=ids)


def run_filters(w):
    orc = O.CPUPath("oracle")
    return np.array([orc.pf_ar1(int(w["N"][k]), w["y"][k], w["phi"][k], w["sx"][k], w["sy"][k], w["sd0"][k],
                                (int(w["ids"][k]), 11), (int(w["ids"][k]), 12), record=False)["loglik"]
                     for k in range(len(w["N"]))])


def fill(rank, n=4096):
    orc = O.CPUPath("oracle")
    return orc.rand(O.Engine.make(O.PHILOX4X32, key=(42,), ctr=shard.rng_counter(rank)), n).astype(np.int64)


def _rank_work(rank, world, port, F, T, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        first, last = shard.filter_range(rank, F)
        w = cpu_workload(last - first, T, 1234, first)
        ll = torch.from_numpy(run_filters(w))
        words = torch.from_numpy(fill(rank))
        lls = [torch.zeros_like(ll) for _ in range(world)]
        ws = [torch.zeros_like(words) for _ in range(world)]
        dist.all_gather(lls, ll)
        dist.all_gather(ws, words)
        units = float(w["N"].astype(np.float64).sum()) * T
        rate, _ = shard.job_rate(units, 1.0 + rank, world)
        if rank == 0:
            q.put((torch.cat(lls).numpy(), torch.stack(ws).numpy(), rate))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reassemble_the_single_process_run():
    world, F, T = 2, 3, 20
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_work, args=(r, world, port, F, T, q)) for r in range(world)]
    for p in procs:
        p.start()
    ll, words, rate = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    whole = cpu_workload(world * F, T, 1234, 0)
    want = run_filters(whole)
    assert np.array_equal(ll, want)  # bit-identical: the same filters, keys and observations
    for r in range(world):
        assert np.array_equal(words[r], fill(r))
    assert not np.array_equal(words[0], words[1])  # disjoint counter ranges
    units = float(whole["N"].astype(np.float64).sum()) * T
    assert rate == pytest.approx(units / 2.0)  # all units over the slower rank's 2 s
