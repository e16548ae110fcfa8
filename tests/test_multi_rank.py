"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (the path
runs replicas, one image per rank, with no collective on the data path;
only the timing is reduced).  The whole-job rate must use the slowest
rank's time."""

import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import sys
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
        t = bench.max_over_ranks(local_ms, torch.device("cpu"), world)
        rate = bench.job_rate(100, world, t / 1e3)
        out[rank] = (t, rate)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_gloo():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2,
                       join=True, start_method="spawn")
    assert out[0][0] == pytest.approx(15.0) and out[1][0] == pytest.approx(15.0)
    # 2 ranks x 100 units in the slowest rank's 15 ms
    assert out[0][1] == pytest.approx(200 / 0.015)


def test_single_rank_needs_no_process_group():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, 1) == 3.5
    assert bench.job_rate(10, 1, 2.0) == 5.0
