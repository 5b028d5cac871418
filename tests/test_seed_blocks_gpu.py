"""The block seeding pass (points whose disk holds many critical-curve source
points) gives the same seeds and results as the one-warp pass, bit for bit,
and both match the reference on such points.

The heavy points put a planet's whole planetary caustic inside the source
disk: every critical source inside the disk gets the reference's caustic
probes, which is where the block pass takes over.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

pytestmark = pytest.mark.gpu


def _checker():
    from oracle.oracle import Oracle, Reference, have_reference
    return Reference() if have_reference() else Oracle()


def _heavy_points():
    """Sources centred on a planetary caustic, with disks that contain it."""
    from oracle.oracle import Oracle
    orc = Oracle()
    rows = []
    for s, q in ((1.3, 1.0e5), (0.8, 2.0e4), (1.6, 5.0e4)):
        br, _, _ = orc.caustic_cache(s, q, 512)
        pts = br.reshape(-1, 2)
        r = np.hypot(pts[:, 0], pts[:, 1])
        far = pts[r > 0.5 * (r.min() + r.max())]
        # the cluster farthest from the origin (one of two for s < 1)
        far = far[np.argsort(-far[:, 1])][: max(1, len(far) // 2)] if s < 1.0 else far
        c = far.mean(axis=0)
        extent = np.max(np.hypot(far[:, 0] - c[0], far[:, 1] - c[1]))
        for rho in (1.3 * extent, 2.5 * extent):
            rows.append((s, q, c[0], c[1], rho))
    return np.array(rows)


def _run(ctx, rows, grid, nbin, c, after):
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs, LimbDarkening, Options, PS_EXACT, PS_ON_DEVICE
    L = ctx._L
    assert L.lcbi_gpu_set_seed_block_after(ctx.handle, after) == 0
    st = Options(inverse_ray_grid=grid, nbin=nbin).fs_settings(LimbDarkening.linear(c))
    st.kinji_threshold = 1e18
    st.hex_threshold = 0.0
    st.adaptive_hex_threshold = 0.0
    sts = (LcbiStructs.FsSettings * 1)(st)
    pts = np.zeros(len(rows), dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    out = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
    ctx.check(L.lcbi_gpu_binary_mag(ctx.handle, sts, 1, None, 0, len(rows), pts.ctypes.data, out.ctypes.data, 0),
              "lcbi_gpu_binary_mag")
    return out, st


@pytest.mark.parametrize("grid", ["cartesian", "polar"])
def test_block_seeding_matches_warp_seeding_and_reference(grid):
    from lcbinint_b200 import _lib
    from oracle.oracle import default_settings
    rows = _heavy_points()
    ctx = _lib.Context(0)
    nbin, c = 30, 0.5
    warp, _ = _run(ctx, rows, grid, nbin, c, 0)
    block, _ = _run(ctx, rows, grid, nbin, c, 1)
    default, _ = _run(ctx, rows, grid, nbin, c, 32)
    assert (warp["status"] == 0).all()
    assert (warp["seed_count"] > 0).all()
    assert block.tobytes() == warp.tobytes()
    assert default.tobytes() == warp.tobytes()
    ref = _checker()
    mode = {"cartesian": 1, "polar": 2}[grid]
    R, _ = ref.inverse_ray(default_settings(source_bins=nbin, finite_mode=mode, limb_darkening_c=c),
                           rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4])
    A = warp["magnification"]
    if grid == "cartesian":
        assert np.array_equal(A.view(np.int64), R.view(np.int64)), (A, R)
    else:
        # the polar sum is exact (128-bit fixed point): same cells, the reference's running sum within 1e-12
        assert np.allclose(A, R, rtol=1e-12, atol=0), (A, R)


def test_block_seeding_on_mixed_batch():
    """A 256-point slice of the 4,096-point fs_batch: every point that meets a
    critical source inside its disk seeded on a block, against one warp each."""
    import bench
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs, PS_EXACT, PS_ON_DEVICE
    rows = bench.fs_batch_workload(seed=6)
    rows = rows[np.random.default_rng(13).permutation(len(rows))[:256]]
    settings, sidx = bench.fs_settings_for(rows)
    st = (LcbiStructs.FsSettings * len(settings))(*settings)
    pts = np.zeros(len(rows), dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    pts["settings"] = sidx
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    ctx = _lib.Context(0)
    outs = []
    for after in (0, 1):
        assert ctx._L.lcbi_gpu_set_seed_block_after(ctx.handle, after) == 0
        out = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
        ctx.check(ctx._L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), None, 0, len(rows), pts.ctypes.data,
                                             out.ctypes.data, 0), "lcbi_gpu_binary_mag")
        outs.append(out)
    assert (outs[0]["status"] == 0).all()
    assert outs[1].tobytes() == outs[0].tobytes()
