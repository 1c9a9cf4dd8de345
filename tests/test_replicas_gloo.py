"""The multi-GPU host logic of bench.py on CPU with two gloo ranks: one partition job does not
shard, so replicas time independently and the job's time is the maximum over ranks; independent
batch jobs shard across ranks with no collective on the data path."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.barrier_max(world, 10.0 * (rank + 1))
        shards = bench.shard_jobs([5, 9, 1, 7, 3, 3, 8], world)
        out.put((rank, t, shards))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_shards_agree():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    times = {r: t for r, t, _ in res}
    assert times == {0: 20.0, 1: 20.0}  # every rank sees the slowest replica's time
    shards = [s for _, _, s in res]
    assert shards[0] == shards[1]  # the same assignment on every rank


def test_shards_cover_every_job_once_and_balance():
    sizes = [int(x) for x in (1e3, 5e4, 2e5, 7e3, 9e4, 3e5, 1e4, 6e4, 4e4)]
    for world in (1, 2, 3, 8):
        shards = bench.shard_jobs(sizes, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in s) for s in shards]
        if world <= len(sizes):
            assert max(loads) - min(loads) <= max(sizes)
