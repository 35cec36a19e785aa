"""Segments across ranks (host logic): partitioning, max-over-ranks timing and
the gather of results, with two gloo ranks on the CPU."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from spikesorting_fullpursuit_b200.parallel import distributed as D  # noqa: E402


def test_partition_covers_every_segment_once_and_balances():
    rng = np.random.default_rng(5)
    costs = rng.integers(1, 1000, size=97).tolist()
    for world in (1, 2, 3, 8):
        shares = D.partition_segments(costs, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shares]
        # greedy longest-first: no rank exceeds the mean by more than the largest segment
        assert max(loads) <= sum(costs) / world + max(costs)
        assert shares == D.partition_segments(costs, world)       # deterministic
    assert D.partition_segments([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        D.partition_segments([1], 0)


def test_without_a_process_group_everything_runs_here():
    segs = [(np.zeros((2, 10 + i), np.float32), {}, {"templates": np.zeros((3, 4))}, 1) for i in range(5)]
    out = D.sort_segments_distributed(segs, runner=lambda v, si, m, nmax: v.shape[1])
    assert out == [10, 11, 12, 13, 14]
    assert D.max_over_ranks(3.5) == 3.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        segs = [(np.full((2, 5 + i), float(i), np.float32), {"i": i}, {"templates": np.zeros((1 + i % 3, 4))}, i)
                for i in range(11)]
        ran = []

        def runner(v, si, m, nmax, scale=1):
            ran.append(si["i"])
            return (si["i"], float(v.sum()) * scale, nmax)

        out = D.sort_segments_distributed(segs, runner=runner, scale=2)
        t = D.max_over_ranks(10.0 + rank, device="cpu")
        q.put((rank, ran, out, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_gather():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(world):
        rank, ran, out, t = q.get(timeout=120)
        got[rank] = (ran, out, t)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ran0, out0, t0 = got[0]
    ran1, out1, t1 = got[1]
    assert sorted(ran0 + ran1) == list(range(11)) and not set(ran0) & set(ran1)
    assert out1 is None
    assert out0 == [(i, 2.0 * i * 2 * (5 + i), i) for i in range(11)]
    assert t0 == t1 == 11.0
