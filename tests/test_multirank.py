"""The multi-GPU timing path of the bench on CPU: two `gloo` ranks, each
with its own step time, agree on the slowest rank's time, and the whole-job
throughput counts every rank's replica.  (On GPUs the same helper reduces
over NCCL; the bench runs one independent replica per GPU: no data
collective.)"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        my_ms = 10.0 + 5.0 * rank
        t = bench.max_over_ranks(my_ms, world, "cpu")
        out[rank] = (t, bench.job_throughput(1000, 20, world, t))
    finally:
        torch.distributed.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    assert res[0] == res[1]
    t, v = res[0]
    assert t == 15.0
    assert v == pytest.approx(1000 * 20 * 2 / 15e-3)


def test_one_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(7.5, 1, "cpu") == 7.5
    assert bench.job_throughput(10, 4, 1, 2.0) == pytest.approx(20000.0)
