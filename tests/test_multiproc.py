"""Multi-process host logic of bench.py on CPU: two gloo ranks, 127.0.0.1."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = [120.0, 95.0][rank]
    rays = [1000, 3000][rank]
    out = bench.reduce_over_ranks(ms, rays, world, "cpu")
    seeds = [None] * world
    dist.all_gather_object(seeds, bench.replica_seed(1, rank))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out, seeds))


def test_two_rank_reduction_and_replica_seeds():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, (ms, rays), seeds in res:
        assert ms == 120.0 and rays == 4000.0  # max time, total rays over ranks
        assert seeds == [1, 2]                 # distinct replicas (weak scaling)


def test_single_rank_passthrough():
    import bench
    assert bench.reduce_over_ranks(5.0, 7, 1, "cpu") == (5.0, 7.0)
