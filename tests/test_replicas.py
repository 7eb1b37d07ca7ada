"""Replica plumbing on CPU: world-size-2 gloo ranks (no GPU)."""

from __future__ import annotations

import os
import socket

import pytest

from beamz_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        items = list(range(11))
        mine = replicas.shard(items, rank, world)
        elapsed = 1.0 + rank  # the slowest rank defines the job time
        t = replicas.max_over_ranks(elapsed)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out.put((rank, t, sorted(sum(gathered, [])), replicas.aggregate_rate(len(mine), t, world)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_shard_and_time_by_the_slowest_rank():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, union, rate in results:
        assert t == 2.0
        assert union == list(range(11))
    assert {r for r, *_ in results} == {0, 1}


def test_single_process_helpers():
    assert replicas.shard(list("abcde"), 1, 2) == ["b", "d"]
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.aggregate_rate(10, 2.0, 4) == 20.0
