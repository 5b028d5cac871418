"""The second Cartesian pass runs on a side stream beside the polar passes
unless stage timing is on; both orders give bit-identical results.

A mixed batch (Cartesian and polar points, nbin 20-200, linear limb
darkening) with a small cell budget sends many Cartesian points to the second
pass, so the side-stream blocks and the polar tile flood share the GPU.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

pytestmark = pytest.mark.gpu


def test_overlapped_second_pass_matches_serial_order():
    import bench
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs, PS_EXACT, PS_ON_DEVICE
    rows = bench.fs_batch_workload(seed=3)
    rows = rows[np.random.default_rng(11).permutation(len(rows))[:384]]
    settings, sidx = bench.fs_settings_for(rows)
    st = (LcbiStructs.FsSettings * len(settings))(*settings)
    pts = np.zeros(len(rows), dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    pts["settings"] = sidx
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    ctx = _lib.Context(0)
    L = ctx._L
    assert L.lcbi_gpu_set_cell_budget(ctx.handle, 1 << 14) == 0

    def run(timing):
        assert L.lcbi_gpu_set_timing(ctx.handle, timing) == 0
        out = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
        ctx.check(L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), None, 0, len(rows), pts.ctypes.data,
                                        out.ctypes.data, 0), "lcbi_gpu_binary_mag")
        return out

    serial = run(1)
    stage_ms = np.zeros(8)
    stage_n = np.zeros(8, dtype=np.int64)
    L.lcbi_gpu_stage_times(ctx.handle, _lib.ptr(stage_ms), _lib.ptr(stage_n), 8)
    overlapped = [run(0) for _ in range(2)]
    assert (serial["status"] == 0).all()
    methods = serial["method"]
    assert (methods == 2).any() and (methods == 3).any()
    # both Cartesian passes and the polar stage ran under timing
    assert stage_n[3] >= 2 and stage_n[4] >= 2
    for r in overlapped:
        assert r.tobytes() == serial.tobytes()


def test_workspace_resize_keeps_second_pass_results():
    """Changing the first-pass warps per SM restarts the scan epoch; the
    second-pass scratch is cleared with it, so tags of earlier scans never
    pass for the current one.  The batch is permuted between calls, so the
    second-pass blocks take other points than before the change."""
    import bench
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs, PS_EXACT, PS_ON_DEVICE
    rows = bench.fs_batch_workload(seed=4)
    rows = rows[np.random.default_rng(12).permutation(len(rows))[:192]]
    settings, sidx = bench.fs_settings_for(rows)
    st = (LcbiStructs.FsSettings * len(settings))(*settings)

    def points(order):
        r = rows[order]
        pts = np.zeros(len(r), dtype=FS_POINT_DTYPE)
        pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = r[:, 0], r[:, 1], r[:, 2], r[:, 3], r[:, 4]
        pts["settings"] = sidx[order]
        pts["flags"] = PS_EXACT | PS_ON_DEVICE
        return pts

    def run(ctx, order):
        pts = points(order)
        out = np.zeros(len(pts), dtype=FS_RESULT_DTYPE)
        ctx.check(ctx._L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), None, 0, len(pts), pts.ctypes.data,
                                             out.ctypes.data, 0), "lcbi_gpu_binary_mag")
        back = np.empty_like(out)
        back[order] = out
        return back

    ident = np.arange(len(rows))
    fresh = run(_lib.Context(0), ident)
    ctx = _lib.Context(0)
    rng = np.random.default_rng(5)
    for _ in range(3):
        run(ctx, rng.permutation(len(rows)))
    assert ctx._L.lcbi_gpu_set_workspace(ctx.handle, 4, 0, 0) == 0
    for _ in range(2):
        got = run(ctx, rng.permutation(len(rows)))
        assert got.tobytes() == fresh.tobytes()


def test_early_block_routing_keeps_results():
    """Cartesian points predicted to need many times the first pass's cell
    budget run on blocks from the start, beside the first pass.  Routing
    changes where a point runs, not what it returns: no routing (budget 0,
    every point on its warp), heavy routing (a small budget, so the 32 largest
    predicted points go early) and the default give the same bytes."""
    import bench
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs, PS_EXACT, PS_ON_DEVICE
    rows = bench.fs_batch_workload(seed=7)
    rows = rows[rows[:, 7] <= 100]  # keep every point small enough for one warp without a budget
    rows = rows[np.random.default_rng(14).permutation(len(rows))[:320]]
    settings, sidx = bench.fs_settings_for(rows)
    st = (LcbiStructs.FsSettings * len(settings))(*settings)
    pts = np.zeros(len(rows), dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    pts["settings"] = sidx
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    outs = {}
    for budget in (0, 1 << 12, 1 << 19):
        ctx = _lib.Context(0)
        assert ctx._L.lcbi_gpu_set_cell_budget(ctx.handle, budget) == 0
        out = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
        ctx.check(ctx._L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), None, 0, len(rows), pts.ctypes.data,
                                             out.ctypes.data, 0), "lcbi_gpu_binary_mag")
        outs[budget] = out
    base = outs[0]
    assert (base["status"] == 0).all()
    assert (base["method"] == 2).any()
    for budget in (1 << 12, 1 << 19):
        assert outs[budget].tobytes() == base.tobytes(), budget


def test_early_helpers_match_the_early_pass_alone():
    """Once the Cartesian passes on the side stream are done, that stream's
    blocks join the early block pass of the largest points and take the units
    it has not started.  With eight second-pass blocks the early pass also has
    eight blocks, so the 4,096-point batch leaves the joining blocks most of
    the early units; the results must be the bytes of the early pass alone."""
    import bench
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs, PS_EXACT, PS_ON_DEVICE
    rows = bench.fs_batch_workload(seed=1)
    settings, sidx = bench.fs_settings_for(rows)
    st = (LcbiStructs.FsSettings * len(settings))(*settings)
    pts = np.zeros(len(rows), dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    pts["settings"] = sidx
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    ctx = _lib.Context(0)
    L = ctx._L
    assert L.lcbi_gpu_set_workspace(ctx.handle, 0, 8, 0) == 0

    def run(helpers):
        assert L.lcbi_gpu_set_early_helpers(ctx.handle, helpers) == 0
        out = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
        ctx.check(L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), None, 0, len(rows), pts.ctypes.data,
                                        out.ctypes.data, 0), "lcbi_gpu_binary_mag")
        return out

    alone = run(0)
    assert (alone["status"] == 0).all()
    for _ in range(2):
        assert run(1).tobytes() == alone.tobytes()
