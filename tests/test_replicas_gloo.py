"""Multi-GPU runs are replicas (the path has no exchange step): `bench.py --gpus N` under torch.distributed
runs one independent solve per rank and reports the slowest rank's time. Checked here with two gloo ranks on
the CPU: both ranks take the maximum, and the job's throughput counts every replica's cells."""
import datetime
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    dist.barrier()
    out[rank] = ms
    dist.destroy_process_group()


def test_replicas_report_the_slowest_rank():
    sys.path.insert(0, ROOT)
    import bench
    world = 2
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        got = dict(out)
    assert got == {0: 15.0, 1: 15.0}
    assert bench.max_over_ranks(7.5, None, "cpu") == 7.5
    assert bench.job_throughput(160000, 200, world, 35.0) == pytest.approx(160000 * 200 * 2 / 0.035)
