"""The multi-GPU path's host logic (replicas, max-over-ranks timing) on two gloo ranks on the CPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from toaster_b200.replicas import job_throughput, max_over_ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_seconds = 1.0 + rank  # the slower rank sets the job time
        job = max_over_ranks(local_seconds)
        out[rank] = (job, job_throughput(1_000_000, 4, world, job))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1]
    job, mpaths = out[0]
    assert job == 2.0
    assert mpaths == pytest.approx(2 * 1_000_000 * 4 / 2.0 / 1e6)


def test_single_process_needs_no_group():
    assert max_over_ranks(3.5) == 3.5
    with pytest.raises(ValueError):
        job_throughput(1, 1, 1, 0.0)
