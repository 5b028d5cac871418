"""lcbi_gpu_autotune: the launch shapes it picks come from its candidate sets,
stay on the context, and change no result (bit-identical magnifications)."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results_and_picks_a_candidate():
    import bench
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs, PS_EXACT, PS_ON_DEVICE
    rows = bench.fs_batch_workload(seed=1)
    rows = rows[np.random.default_rng(8).permutation(len(rows))[:256]]
    settings, sidx = bench.fs_settings_for(rows)
    st = (LcbiStructs.FsSettings * len(settings))(*settings)
    pts = np.zeros(len(rows), dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    pts["settings"] = sidx
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    ctx = _lib.Context(0)
    L = ctx._L
    plain = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
    ctx.check(L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), None, 0, len(rows), pts.ctypes.data,
                                    plain.ctypes.data, 0), "lcbi_gpu_binary_mag")
    tuned = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
    shape = np.zeros(3, dtype=np.int32)
    best = C.c_double(0.0)
    ctx.check(L.lcbi_gpu_autotune(ctx.handle, st, len(settings), None, 0, len(rows), pts.ctypes.data,
                                  tuned.ctypes.data, 0, shape.ctypes.data, C.byref(best)), "lcbi_gpu_autotune")
    assert best.value > 0.0
    assert shape[1] in (4, 8) and shape[0] >= 1 and shape[2] >= 1
    after = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
    ctx.check(L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), None, 0, len(rows), pts.ctypes.data,
                                    after.ctypes.data, 0), "lcbi_gpu_binary_mag")
    for r in (tuned, after):
        assert r.tobytes() == plain.tobytes()
