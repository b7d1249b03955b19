"""The replicas-only multi-process path of bench.py on CPU (gloo, world size 2).

The hot path does not shard: with N GPUs every rank advances its own replica
(its own Philox stream), the job's time is the slowest rank's and the value is
the sum over ranks.  This exercises that host logic with two gloo ranks."""
import multiprocessing as mp
import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as td

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        ms = bench.max_over_ranks(10.0 + 5.0 * rank, "cpu", True)
        value = bench.job_rate(1000, 10, world, ms / 1e3)
        q.put((rank, ms, value, bench.replica_stream(rank)))
        # the reference arm: ranks other than 0 return without work
        if rank != 0:
            class A:
                steps, warmup, gpus, workload = 1, 3, world, "triangular1024_thermal"

            assert bench.run_reference(A(), rank, world) is None
        td.barrier()
    finally:
        td.destroy_process_group()


def test_two_rank_replicas_reduce_to_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [15.0, 15.0]              # max over ranks, on every rank
    assert out[0][2] == pytest.approx(1000 * 10 * 2 / 15e-3)  # whole-job rate
    assert out[0][3] != out[1][3]                            # independent noise streams
