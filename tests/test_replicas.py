"""The multi-GPU path is replicas (independent solves per rank, no data-path
collective): the job's time is the slowest rank's and its work the sum. The
aggregation runs here as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    times, cells = bench.reduce_over_ranks([1.0 + rank, 10.0 - rank], 1000 * (rank + 1), dist, "cpu")
    out[rank] = (times, cells)
    dist.barrier()
    dist.destroy_process_group()


def test_slowest_rank_and_summed_work():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        times, cells = out[r]
        assert times == [2.0, 10.0]
        assert cells == 3000.0
