"""Replica plumbing of the multi-GPU benchmark, exercised with world_size 2 over gloo on the CPU."""
import os
import socket

import torch.multiprocessing as mp

import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        elapsed = 1.0 + rank  # rank 1 is the slow one
        m = replicas.max_over_ranks(elapsed)
        seeds = [replicas.pair_seed(rank, i) for i in range(3)]
        out[rank] = (m, seeds, replicas.aggregate_rate(16, world, m))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_distinct_work_with_gloo():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.0          # every rank sees the slowest rank's time
    assert set(res[0][1]).isdisjoint(res[1][1])   # ranks solve distinct pairs
    assert res[0][2] == 16 * 2 / 2.0              # whole-job pairs / max time


def test_single_process_is_identity():
    assert replicas.max_over_ranks(3.5) == 3.5
