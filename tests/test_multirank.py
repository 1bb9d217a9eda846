"""The multi-rank host logic of bench.py on CPU: gloo, world size 2, one process per rank.  Every
rank takes the same collective steps; the job time is the maximum over ranks."""
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

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    try:
        out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank, world)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert out[0] == out[1] == 15.0


def test_max_over_ranks_single():
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5
