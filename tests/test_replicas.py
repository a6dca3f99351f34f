"""The multi-GPU path of bench.py is replicas only: every rank solves its own
copy of the workload, and the only collectives are the barrier around the
timed region and the max over ranks of its duration. Those run here as two
gloo ranks on the CPU (127.0.0.1), as torchrun would start them."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        bench.barrier(world)
        # each rank times its own replica; the job's time is the slowest rank's
        ms = 10.0 + 5.0 * rank
        got = bench.max_over_ranks(ms, world, torch.device("cpu"))
        # the reference arm runs on rank 0 only; the other ranks return nothing
        class A:
            m, n, steps, warmup = 600, 400, 1, 0
        ref = bench.run_reference(A, world, rank) if rank != 0 else "skipped"
        bench.barrier(world)
        out[rank] = (got, ref)
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_max_over_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    assert res[0][0] == pytest.approx(15.0) and res[1][0] == pytest.approx(15.0)
    assert res[1][1] is None
