"""The multi-GPU path is replicas only: every rank searches the same sources on its
own GPU, and the job's time is the slowest rank's.  The rank combination of
bench.py is exercised here with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow replica
        slowest = bench.max_over_ranks(ms, dist, device="cpu")
        value = bench.replica_gteps(1e9, world, slowest * 1e-3)
        out[rank] = (slowest, value)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    slowest, value = res[0]
    assert slowest == 15.0
    assert value == pytest.approx(2 * 1e9 / 15e-3 / 1e9)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_gteps(2e9, 1, 1.0) == pytest.approx(2.0)
