"""The multi-GPU form of the benchmark is N independent replicas (no data
moves between ranks): the job's time is the slowest rank's, and the
throughput counts every rank's steps.  Two gloo ranks on the CPU check the
reduction the benchmark uses."""
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
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    seconds = 1.0 + rank  # rank 1 is the slow one
    out[rank] = (bench.max_over_ranks(seconds), bench.replica_value(5, seconds))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    world, port = 2, _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        for r in range(world):
            slow, value = out[r]
            assert slow == 2.0
            assert value == pytest.approx(world * 5 / 2.0)
