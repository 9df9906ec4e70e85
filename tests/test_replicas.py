"""Replica scaling host logic on two gloo ranks (CPU): disjoint frames per
rank, the job time is the slowest rank's time on every rank, and the job rate
counts every rank's units. No GPU and no collective on the data path."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from bevy_strand_rasterizer_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        frames = [replicas.frame_index(rank, k) for k in range(50)]
        elapsed = 1.0 + 0.5 * rank  # rank 1 is the slow one
        slowest = replicas.max_over_ranks(elapsed)
        rate = replicas.job_rate(1000.0, world, slowest)
        out.put((rank, frames, slowest, rate))
    finally:
        dist.destroy_process_group()


def test_two_replicas():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by_rank = {r: (frames, slowest, rate) for r, frames, slowest, rate in results}
    assert set(by_rank[0][0]).isdisjoint(by_rank[1][0])
    for r in range(world):
        assert by_rank[r][1] == pytest.approx(1.5)
        assert by_rank[r][2] == pytest.approx(1000.0 * world / 1.5)


def test_single_process_is_identity():
    assert replicas.max_over_ranks(3.25) == 3.25
    assert replicas.job_rate(10.0, 1, 2.0) == 5.0
