"""bench.py's multi-GPU bookkeeping on CPU: world_size-2 gloo ranks, each timing its own
replica, agree on the max over ranks, and the aggregate is world x bytes / that max."""
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


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, main_ms = bench.max_over_ranks([1.0 + rank, 0.5 + 0.25 * (1 - rank)], world, "cpu")
        e2e, = bench.max_over_ranks([3.0 * (rank + 1)], world, "cpu")
        dist.barrier()
        out[rank] = (ms, main_ms, e2e, bench.aggregate_gbps(world, 1e9, ms))
    finally:
        dist.destroy_process_group()


def test_two_replicas_agree_on_max():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn")
    for r in range(world):
        ms, main_ms, e2e, agg = out[r]
        assert (ms, main_ms, e2e) == (2.0, 0.75, 6.0)
        assert agg == pytest.approx(2 * 1e9 / 2e-3 / 1e9)


def test_single_rank_is_identity():
    assert bench.max_over_ranks([1.5, 2.5], 1, "cpu") == [1.5, 2.5]
    assert bench.aggregate_gbps(1, 8e9, 1.0) == pytest.approx(8000.0)
