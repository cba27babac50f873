"""Multi-GPU scheme of bench.py: independent replicas, one process per GPU,
no data-path collective; the only collective is the MAX over ranks of the
timed duration, which sets the whole-job rate.  Run here with the gloo
backend and two CPU processes."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r pretends its K = 10 timed steps took (1 + r) seconds
        t = bench.max_over_ranks(1.0 + rank, dist, torch.device("cpu"))
        out[rank] = (t, bench.whole_job_rate(world, 10, t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_gloo():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert dict(out) == {0: (2.0, 10.0), 1: (2.0, 10.0)}  # slowest rank: 2 s; 2 x 10 evals / 2 s


def test_single_process_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, None) == 3.5
    assert bench.whole_job_rate(1, 20, 0.5) == 40.0
