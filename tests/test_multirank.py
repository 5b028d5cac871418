"""Multi-process host logic of bench.py's multi-GPU run, on CPU with gloo
(world size 2): each rank runs its own replica batch, and the job's numbers are
the slowest rank's times and the work of all ranks."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        rows = bench.fs_batch_workload(seed=1 + rank)
        maxes, sums = bench.reduce_over_ranks([10.0 * (rank + 1), 3.0 - rank], [len(rows), 100.0 * (rank + 1)],
                                              world, torch.device("cpu"))
        out[rank] = (maxes, sums, float(rows[:, 2].sum()))
    finally:
        dist.destroy_process_group()


def test_replica_reduction_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    port = _free_port()
    # spawn, not fork: the test process may already hold a CUDA context
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for rank in (0, 1):
        maxes, sums, _ = res[rank]
        assert maxes == [20.0, 3.0]
        assert sums == [2 * 4096.0, 300.0]
    # replicas: each rank has its own batch of the same size
    assert res[0][2] != res[1][2]


def test_single_rank_reduction_is_identity():
    import bench
    assert bench.reduce_over_ranks([1.5, 2.0], [7, 8.0], 1, None) == ([1.5, 2.0], [7.0, 8.0])
