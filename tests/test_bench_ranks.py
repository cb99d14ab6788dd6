"""The multi-replica host logic of bench.py on two gloo ranks (CPU): the
timing is the maximum over ranks, every rank sees it, and the whole-job rate
counts every replica's cells."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = [0.25, 0.4][rank]                      # this rank's device seconds
        t = bench.max_over_ranks(local, world, device="cpu")
        out[rank] = (t, bench.whole_job_rate(world, 1000, 10, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_time():
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0][0] == pytest.approx(0.4) and out[1][0] == pytest.approx(0.4)
    assert out[0][1] == pytest.approx(2 * 1000 * 10 / 0.4)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(1.5, 1) == 1.5
    assert bench.whole_job_rate(1, 100, 3, 0.5) == 600
