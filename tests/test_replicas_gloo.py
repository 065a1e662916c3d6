"""The multi-GPU path of bench.py is replicas only: each rank plans independently and the job
time is the maximum device time over ranks, the work the sum.  Checked here with two gloo ranks
on the CPU (no device work)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    t, v = bench.combine_over_ranks(dist, "cpu", 1.0 + rank, 100 * (rank + 1))
    out[rank] = (t, v)
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_combine_max_time_and_summed_work():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0] == res[1] == (2.0, 300.0)


def test_single_process_passthrough():
    import bench

    assert bench.combine_over_ranks(None, "cpu", 1.5, 7) == (1.5, 7.0)
