"""The N > 1 path of the batched workloads on CPU: two gloo ranks, as one
process per GPU would run them.  The ranks' filter ranges and RNG counter
ranges are disjoint and cover the global workload, and the whole-job rate is
the units summed over ranks over the slowest rank's time, with every rank
taking the same collective steps."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

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
