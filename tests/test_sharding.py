"""Case sharding across ranks (the multi-GPU path of bench.py) with gloo ranks on CPU:
every case lands on exactly one rank, and the combined measurements are the sum of the
cases, the max of the durations and the union of the latencies."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from matlab_ufvm_b200 import sharding


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n_total, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = sharding.shard(rank, world, n_total)
        assert mine == [sharding.stream_index(rank, world, k) for k in range(len(mine))]
        converged = len(mine)                      # stands in for this rank's converged cases
        ms = 100.0 + 10.0 * rank                   # stands in for this rank's timed duration
        total = sharding.reduce_sum(converged)
        slowest = sharding.reduce_max(ms)
        everyone = sharding.gather(mine)
        q.put((rank, total, slowest, sorted(everyone)))
    finally:
        dist.destroy_process_group()


def test_shards_partition_the_stream():
    for world in (1, 2, 3, 8):
        seen = []
        for r in range(world):
            seen += sharding.shard(r, world, 1000)
        assert sorted(seen) == list(range(1000))
    with pytest.raises(ValueError):
        sharding.stream_index(2, 2, 0)


def test_batch_seeds_are_distinct_per_rank():
    for world in (1, 2, 4, 8):
        seeds = [sharding.batch_seed(r, world, 2024) for r in range(world)]
        assert seeds[0] == 2024 and len(set(seeds)) == world
    with pytest.raises(ValueError):
        sharding.batch_seed(4, 4, 2024)


def test_two_gloo_ranks_combine_measurements():
    world, n_total = 2, 37
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n_total, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, total, slowest, everyone in out:
        assert total == n_total
        assert slowest == 100.0 + 10.0 * (world - 1)
        assert everyone == list(range(n_total))
