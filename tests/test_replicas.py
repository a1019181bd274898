"""bench.py --gpus N runs N independent replicas: the path does not shard, and the only
cross-rank step is the max of the timings.  Two gloo ranks on the CPU check that step and
the whole-job rate built on it."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took 10 + r seconds for its solves and 20 - r for the e2e ones
        total, e2e = bench.max_over_ranks([10.0 + rank, 20.0 - rank], dist, "cpu")
        out[rank] = (total, e2e, bench.whole_job_rate(3, 2, world, total))
    finally:
        dist.destroy_process_group()


def test_replica_timings_take_the_slowest_rank():
    world, port = 2, _free_port()
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        results = dict(out)
    for rank in range(world):
        total, e2e, rate = results[rank]
        assert total == 11.0 and e2e == 20.0
        assert rate == pytest.approx(3600.0 * 3 * 2 * world / 11.0)


def test_without_a_process_group_values_pass_through():
    import bench
    assert bench.max_over_ranks([1.5, 2.5], None, "cpu") == [1.5, 2.5]
    assert bench.whole_job_rate(3, 1, 1, 10.8) == pytest.approx(1000.0)
