"""Multi-GPU host logic, on CPU (gloo, world size 2): one finite-source batch
split over the ranks by LPT on estimated lattice cells
(lcbinint_b200.shard.lpt_partition), each rank's results gathered into input
order on every rank (shard.gather_results), and the bench's reduction of the
job's numbers (the slowest rank's time, the work of all ranks)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _costs(n, seed):
    """Cell counts spread like the finite-source batch's: 1e3 to 1e7."""
    return np.exp(np.random.default_rng(seed).uniform(np.log(1e3), np.log(1e7), n))


def test_lpt_partition_is_complete_ordered_deterministic_and_balanced():
    from lcbinint_b200.shard import lpt_partition
    for n, m, seed in ((4096, 2, 1), (8192, 8, 2), (7, 3, 3), (3, 5, 4), (0, 2, 5)):
        c = _costs(n, seed)
        parts = lpt_partition(c, m)
        assert len(parts) == m
        allidx = np.concatenate(parts) if n else np.zeros(0, dtype=np.int64)
        assert np.array_equal(np.sort(allidx), np.arange(n))  # every point exactly once
        for p in parts:
            assert np.all(np.diff(p) > 0)  # input order inside a share
        again = lpt_partition(c.copy(), m)
        assert all(np.array_equal(a, b) for a, b in zip(parts, again))  # same on every rank
        if n:
            loads = np.array([c[p].sum() for p in parts])
            bound = max(c.sum() / m, c.max())  # no split beats this
            assert loads.max() <= (4.0 / 3.0) * bound  # Graham's LPT guarantee
    # Equal costs: ties go by index and to the lowest part.
    parts = lpt_partition(np.ones(5), 2)
    assert [p.tolist() for p in parts] == [[0, 2, 4], [1, 3]]
    with pytest.raises(ValueError):
        lpt_partition([1.0, -1.0], 2)
    with pytest.raises(ValueError):
        lpt_partition([1.0], 0)


def test_point_costs_follow_the_cell_estimate():
    from lcbinint_b200.api import FS_POINT_DTYPE, LimbDarkening, Options
    from lcbinint_b200.shard import lpt_partition, point_costs
    st = [Options(nbin=20).fs_settings(LimbDarkening()), Options(nbin=200).fs_settings(LimbDarkening())]
    pts = np.zeros(4, dtype=FS_POINT_DTYPE)
    pts["settings"] = [0, 1, 0, 1]
    c = point_costs(pts, st, a_ps=np.array([1.0, 3.0, 0.2, 1000.0]))
    assert np.allclose(c, np.pi * np.array([400.0, 3 * 40000.0, 400.0, 1000 * 40000.0]))
    # The largest point gets a rank to itself.
    assert lpt_partition(c, 2)[0].tolist() == [3]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    import bench
    from lcbinint_b200.api import FS_RESULT_DTYPE
    from lcbinint_b200.shard import gather_results, lpt_partition
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        n = 1000
        parts = lpt_partition(_costs(n, 9), world)
        mine = parts[rank]
        # Each rank's stand-in results for its share: values that name the point.
        local = np.zeros(len(mine), dtype=FS_RESULT_DTYPE)
        local["magnification"] = 1.5 * mine
        local["method"] = mine % 4
        local["seed_count"] = rank
        full = gather_results(local, parts, n)
        maxes, sums = bench.reduce_over_ranks([10.0 * (rank + 1), 3.0 - rank], [len(mine), 100.0 * (rank + 1)],
                                              world, torch.device("cpu"))
        out[rank] = (full.tobytes(), [p.tolist() for p in parts], maxes, sums)
    finally:
        dist.destroy_process_group()


def test_sharded_batch_gathers_in_input_order_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    from lcbinint_b200.api import FS_RESULT_DTYPE
    port = _free_port()
    # spawn, not fork: the test process may already hold a CUDA context
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    n = 1000
    full0 = np.frombuffer(res[0][0], dtype=FS_RESULT_DTYPE)
    full1 = np.frombuffer(res[1][0], dtype=FS_RESULT_DTYPE)
    assert full0.tobytes() == full1.tobytes()  # every rank holds the whole batch
    assert np.array_equal(full0["magnification"], 1.5 * np.arange(n))
    assert np.array_equal(full0["method"], np.arange(n) % 4)
    owner = np.zeros(n, dtype=np.int32)
    owner[res[0][1][1]] = 1
    assert np.array_equal(full0["seed_count"], owner)
    assert res[0][1] == res[1][1]  # the same partition on both ranks
    for rank in (0, 1):
        maxes, sums = res[rank][2], res[rank][3]
        assert maxes == [20.0, 3.0]  # the slowest rank's time
        assert sums == [float(n), 300.0]  # the work of all ranks


def test_single_rank_reduction_is_identity():
    import bench
    assert bench.reduce_over_ranks([1.5, 2.0], [7, 8.0], 1, None) == ([1.5, 2.0], [7.0, 8.0])
