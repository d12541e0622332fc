"""Replica sharding over a real two-rank gloo process group on CPU: every CPI is owned by
exactly one rank and the timing reduction returns the slowest rank's time."""
from __future__ import annotations

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    from zkx_dev_b200.replicas import max_over_ranks, shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cpis = list(range(11))
        mine = shard(cpis, rank, world)
        counts = torch.zeros(len(cpis), dtype=torch.int64)
        for c in mine:
            counts[c] += 1
        dist.all_reduce(counts)
        timing = max_over_ranks([1.0 + rank, 5.0 - rank], dist)
        out.put((rank, counts.tolist(), timing))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_cover_every_cpi_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, counts, timing in results:
        assert counts == [1] * 11
        assert timing == [2.0, 5.0]


def test_shard_single_rank_and_bad_arguments():
    from zkx_dev_b200.replicas import shard
    assert shard(list(range(5)), 0, 1) == [0, 1, 2, 3, 4]
    with pytest.raises(ValueError):
        shard([1], 2, 2)
