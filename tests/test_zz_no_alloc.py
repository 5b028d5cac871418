"""lcbi_gpu_binary_mag_noalloc through the C ABI against lcbi_gpu_binary_mag.

The no-allocation entry point keeps all of its working memory in one fixed
device array, so the test calls it twice in a row on the same inputs (the
second call must not see anything the first left behind) and requires both
results to equal, field for field and bit for bit, what the workspace entry
point returns for the same points.  The file name sorts last so the test also
runs after every other GPU test in the same process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    from lcbinint_b200 import _lib
    return _lib, _lib.lib()


def _points(s, q, n, seed):
    """Source positions around the caustic of (s, q): the decision tree sends
    them to every method (point source, hexadecapole, Cartesian, polar)."""
    from oracle.oracle import Oracle
    rng = np.random.default_rng(seed)
    br, _, _ = Oracle().caustic_cache(s, q, 256)
    pts = br.reshape(-1, 2)
    rho = np.exp(rng.uniform(np.log(2e-3), np.log(2e-2), n))
    p = pts[rng.integers(len(pts), size=n)] + rng.normal(0.0, 1.0, (n, 2)) * rho[:, None] * rng.choice(
        [0.5, 3.0, 30.0], size=(n, 1))
    return p[:, 0].copy(), p[:, 1].copy(), rho


def _settings(mode, c):
    from lcbinint_b200.api import LcbiStructs
    return LcbiStructs.FsSettings(
        source_bins=24, caustic_bins=1400, grid_ratio=4.0, polar_source_bins=0, polar_grid_ratio=0.0,
        finite_mode=mode, kinji_threshold=20.0, hex_threshold=3.0, adaptive_hex_threshold=0.001,
        limb_darkening_c=c, limb_darkening_d=0.0, adaptive_source_bins=0, max_source_bins=400,
        finite_source_tol=0.0, finite_source_reltol=0.0)


def _workspace(ctx, L, st, s, q, y1, y2, rho):
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, PS_EXACT, PS_ON_DEVICE
    n = y1.size
    pts = np.zeros(n, dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = s, q, y1, y2, rho
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    res = np.zeros(n, dtype=FS_RESULT_DTYPE)
    rc = L.lcbi_gpu_binary_mag(ctx.handle, C.byref(st), 1, None, 0, n, pts.ctypes.data, res.ctypes.data, 0)
    ctx.check(rc, "lcbi_gpu_binary_mag")
    return res


def _noalloc(ctx, L, st, s, q, y1, y2, rho):
    import torch
    from lcbinint_b200.api import FS_RESULT_DTYPE
    n = y1.size
    dev = torch.device("cuda", ctx.device)
    d1, d2, dr = (torch.from_numpy(a).to(dev) for a in (y1, y2, rho))
    out = torch.zeros(n * FS_RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)
    rc = L.lcbi_gpu_binary_mag_noalloc(ctx.handle, C.byref(st), s, q, n, d1.data_ptr(), d2.data_ptr(),
                                       dr.data_ptr(), out.data_ptr())
    ctx.check(rc, "lcbi_gpu_binary_mag_noalloc")
    return out.cpu().numpy().view(FS_RESULT_DTYPE)


def _same(a, b):
    for f in ("magnification", "error_estimate"):
        x, y = a[f], b[f]
        assert np.array_equal(np.isnan(x), np.isnan(y)), f
        ok = ~np.isnan(x)
        assert np.array_equal(x[ok].view(np.int64), y[ok].view(np.int64)), \
            f"{f}: {np.sum(x[ok] != y[ok])} of {ok.sum()} differ"
    for f in ("method", "converged", "status", "seed_count"):
        assert np.array_equal(a[f], b[f]), f


@pytest.mark.parametrize("mode,c", [(1, 0.0), (2, 0.5), (4, 0.3)])
def test_noalloc_matches_workspace_entry_point_twice(mode, c):
    _lib_mod, L = _lib()
    ctx = _lib_mod.Context(0)
    try:
        st = _settings(mode, c)
        s, q = 0.9, 1.0 / 0.05
        # 300 points: more than one 256-point pass of the fixed area.
        y1, y2, rho = _points(s, q, 300, seed=mode)
        ref = _workspace(ctx, L, st, s, q, y1, y2, rho)
        want = {1: {0, 1, 2}, 2: {0, 1, 3}, 4: {0, 1, 2, 3}}[mode]
        assert set(np.unique(ref["method"]).tolist()) >= want, np.unique(ref["method"])
        first = _noalloc(ctx, L, st, s, q, y1, y2, rho)
        second = _noalloc(ctx, L, st, s, q, y1, y2, rho)
        _same(first, ref)
        _same(second, ref)
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_the_fixed_area():
    _lib_mod, L = _lib()
    ctx = _lib_mod.Context(0)
    try:
        assert L.lcbi_gpu_binary_mag_noalloc(ctx.handle, C.byref(_settings(1, 0.0)), 0.9, 20.0, 0,
                                             None, None, None, None) == _lib_mod.LCBI_OK
        st = _settings(1, 0.0)
        st.caustic_bins = 4096
        rc = L.lcbi_gpu_binary_mag_noalloc(ctx.handle, C.byref(st), 0.9, 20.0, 0, None, None, None, None)
        assert rc == _lib_mod.LCBI_INVALID_ARGUMENT
        assert b"2048" in L.lcbi_gpu_last_error(ctx.handle)
    finally:
        ctx.close()
