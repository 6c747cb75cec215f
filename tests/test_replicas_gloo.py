"""Replica mode on CPU ranks (gloo, world size 2): whole-job rate from the slowest rank."""
import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from spns_b200.replicas import max_over_ranks, whole_job_rate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    seconds = 2.0 if rank == 1 else 1.0
    m = max_over_ranks(seconds, dist, "cpu")
    out[rank] = whole_job_rate(world, 10, m)
    dist.barrier()
    dist.destroy_process_group()


def test_whole_job_rate_uses_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == pytest.approx(10.0) and out[1] == pytest.approx(10.0)
