"""Replica timing over ranks (bench.py under torchrun): 2 gloo ranks on CPU. Each replica
reports its own device time; the job time is the slowest rank and the value counts every
rank's records."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    local = [100.0, 250.0][rank]
    total, value = bench.combine_ranks(local, records_per_rank=1_000_000, steps=5, world=world,
                                       dist=dist, device="cpu")
    q.put((rank, total, value))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, total, value in out:
        assert total == 250.0
        assert value == pytest.approx(2 * 1_000_000 * 5 / 0.25)


def test_single_rank_needs_no_process_group():
    import bench
    total, value = bench.combine_ranks(50.0, 10, 2, 1)
    assert total == 50.0 and value == pytest.approx(10 * 2 / 0.05)
