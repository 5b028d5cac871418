"""FP32 ray map (lcbi_gpu_set_ray_precision(ctx, 32)) against the bit-exact
FP64 map on forced inverse-ray points of the fs_batch distribution (Cartesian
and polar, nbin 20-200, linear limb darkening): every magnification within
1e-4 relative (the precision the FP32 arm is quoted at), most far closer."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

pytestmark = pytest.mark.gpu


def test_fp32_rays_within_stated_error():
    import bench
    import lcbinint_b200 as lb
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs, PS_EXACT, PS_ON_DEVICE
    rows = bench.fs_batch_workload(seed=1)
    rows = rows[np.random.default_rng(3).permutation(len(rows))[:300]]
    settings, sidx = bench.fs_settings_for(rows)
    st = (LcbiStructs.FsSettings * len(settings))(*settings)
    pts = np.zeros(len(rows), dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    pts["settings"] = sidx
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    ctx = _lib.Context(0)
    L = ctx._L
    out = {}
    for bits in (64, 32):
        assert L.lcbi_gpu_set_ray_precision(ctx.handle, bits) == 0
        res = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
        ctx.check(L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), None, 0, len(rows), pts.ctypes.data,
                                        res.ctypes.data, 0), "lcbi_gpu_binary_mag")
        out[bits] = res
    assert L.lcbi_gpu_set_ray_precision(ctx.handle, 48) == 1
    a64, a32 = out[64]["magnification"], out[32]["magnification"]
    assert np.isfinite(a64).all() and np.isfinite(a32).all()
    assert (out[64]["method"] == out[32]["method"]).all()
    rel = np.abs(a32 / a64 - 1.0)
    assert rel.max() <= 1e-4, rel.max()
    assert np.median(rel) <= 1e-6, np.median(rel)
