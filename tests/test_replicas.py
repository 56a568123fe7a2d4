"""Replica helpers: nnz-balanced partition, and max-over-ranks with two gloo ranks on CPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from psipm_b200.replicas import max_over_ranks, partition_by_nnz


def test_partition_is_a_balanced_cover():
    nnz = [50, 10, 40, 30, 20, 60, 5]
    parts = partition_by_nnz(nnz, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(nnz)))
    loads = [sum(nnz[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(nnz)
    assert partition_by_nnz(nnz, 3) == parts  # deterministic
    assert partition_by_nnz([], 2) == [[], []]
    with pytest.raises(ValueError):
        partition_by_nnz(nnz, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = max_over_ranks(1.5 * (rank + 1))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert dict(out) == {0: 3.0, 1: 3.0}


def test_max_over_ranks_single_process():
    assert max_over_ranks(2.5) == 2.5
