"""Multi-GPU path of the bench (replicas only: independent monolayers, no exchange on the step
path), run as world_size-2 gloo ranks on CPU: the whole-job value is the sum of the ranks' work
over the max of their device times, and every rank agrees on it."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    import bench
    # rank r took (1 + r) s for (10 - r) steps of 100 cells
    value, total = bench.replica_aggregate(1.0 + rank, 10 - rank, 100, world, "cpu")
    out[rank] = (value, total)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_aggregate_two_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    expect_total = 2.0
    expect_value = (10 + 9) * 100 / expect_total
    for r in range(world):
        assert out[r][1] == pytest.approx(expect_total)
        assert out[r][0] == pytest.approx(expect_value)


def test_replica_aggregate_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_aggregate(0.5, 10, 100, 1, "cpu") == (2000.0, 0.5)
