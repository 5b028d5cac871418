"""Bounded device waits, made to run out on purpose without any fault.

The tile-parallel polar flood fill hands tiles between persistent warps
through a FIFO; a warp waiting for its ticket gives up after a bounded number
of polls, stops the flood and leaves its points to the one-block-per-point
second pass.  With the bound lowered to one poll (lcbi_gpu_set_wait_limit),
waits give up as soon as a ticket is not ready: the call must still return
every point's magnification unchanged, report the waits that gave up
(lcbi_gpu_last_wait_timeouts), and the next call with the default bound must
run clean on the same context."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch():
    """Polar points of the finite-source batch with at most about 5e4 azimuthal
    bins, which the second pass takes within its own limits."""
    import bench
    rows = bench.fs_batch_workload(seed=1)
    rows = rows[(rows[:, 6] == 2) & (rows[:, 4] >= 2e-3) & (rows[:, 7] <= 60)]
    return rows[np.random.default_rng(12).permutation(len(rows))[:128]]


def _run(ctx, rows):
    import bench
    from lcbinint_b200.api import FS_RESULT_DTYPE, LcbiStructs
    settings, models, pts = bench.fs_batch_arrays(rows)
    st = (LcbiStructs.FsSettings * len(settings))(*settings)
    res = np.zeros(len(pts), dtype=FS_RESULT_DTYPE)
    ctx.check(ctx._L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), models.ctypes.data, len(models), len(pts),
                                         pts.ctypes.data, res.ctypes.data, 2), "lcbi_gpu_binary_mag")
    n = C.c_int32(-1)
    ctx.check(ctx._L.lcbi_gpu_last_wait_timeouts(ctx.handle, C.byref(n)), "lcbi_gpu_last_wait_timeouts")
    return res, n.value


def _same(a, b):
    assert np.array_equal(a["magnification"].view(np.int64), b["magnification"].view(np.int64))
    for f in ("method", "status", "converged", "seed_count"):
        assert np.array_equal(a[f], b[f]), f


def test_tile_waits_that_run_out_leave_results_unchanged():
    from lcbinint_b200 import _lib
    rows = _batch()
    ctx = _lib.Context(0)
    try:
        base, t0 = _run(ctx, rows)
        assert t0 == 0
        assert (base["status"] == 0).all() and (base["method"] == 3).all()
        ctx.check(ctx._L.lcbi_gpu_set_wait_limit(ctx.handle, 1), "lcbi_gpu_set_wait_limit")
        short, t1 = _run(ctx, rows)
        assert t1 > 0  # waits gave up ...
        _same(short, base)  # ... and the second pass integrated those points the same
        ctx.check(ctx._L.lcbi_gpu_set_wait_limit(ctx.handle, 0), "lcbi_gpu_set_wait_limit")
        again, t2 = _run(ctx, rows)
        assert t2 == 0  # the default bound: a clean call on the same context
        _same(again, base)
    finally:
        ctx.close()
