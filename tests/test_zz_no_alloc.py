"""lcbi_gpu_binary_mag_noalloc through the C ABI against lcbi_gpu_binary_mag.

The no-allocation entry point serves callers that cannot let the library
allocate device memory in the middle of their run (a sampler that has handed
all free memory to its own pool, or one whose other streams must not wait on
a device-wide cudaFree).  All of its working memory is one fixed device array
that every call shares, so the tests here check that:

* results equal, field for field and bit for bit, what the workspace entry
  point returns for the same points, over three calls in a row: a lens model,
  another lens model with other points, then the first again -- so anything
  the fixed array keeps from one call that leaked into the next would show;
* points whose Cartesian scan or polar flood fill outgrows the first pass's
  share of the array (an Einstein ring about the heavier lens) go through the
  four-block second pass and still match;
* past the second pass's limits the point gets status 18 (Cartesian rows) or
  19 (polar segments) and NaN, where the workspace entry point goes on;
* once set up, a call allocates nothing: the device's free memory is the same
  before and after it, and the context's workspaces stay empty;
* requests beyond the fixed array (caustic_bins) are rejected, and adaptive
  refinement is refused.

The file name sorts last so the tests also run after every other GPU test in
the same process; each creates its own context.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RING = (3.0, 1e-6)  # heavier lens at the centre of mass, the lighter one far away


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


def _ring_points(rhos, n_other, seed, offset=1e-4):
    """Sources on the heavier lens of RING (Einstein rings, tens of thousands of
    lattice rows) followed by n_other sources around the lens."""
    rng = np.random.default_rng(seed)
    k = len(rhos)
    y1 = np.concatenate([offset + 1e-5 * np.arange(k), rng.uniform(-1.2, 1.2, n_other)])
    y2 = np.concatenate([np.zeros(k), rng.uniform(-1.2, 1.2, n_other)])
    rho = np.concatenate([np.asarray(rhos, dtype=np.float64),
                          np.exp(rng.uniform(np.log(1e-3), np.log(3e-2), n_other))])
    return y1, y2, rho


def _settings(mode, c, bins=24, **kw):
    from lcbinint_b200.api import LcbiStructs
    st = LcbiStructs.FsSettings(
        source_bins=bins, caustic_bins=1400, grid_ratio=4.0, polar_source_bins=0, polar_grid_ratio=0.0,
        finite_mode=mode, kinji_threshold=20.0, hex_threshold=3.0, adaptive_hex_threshold=0.001,
        limb_darkening_c=c, limb_darkening_d=0.0, adaptive_source_bins=0, max_source_bins=400,
        finite_source_tol=0.0, finite_source_reltol=0.0)
    for k, v in kw.items():
        setattr(st, k, v)
    return st


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


class _Device:
    """Device copies of one call's inputs and its result array."""

    def __init__(self, ctx, y1, y2, rho):
        import torch
        from lcbinint_b200.api import FS_RESULT_DTYPE
        dev = torch.device("cuda", ctx.device)
        self.n = y1.size
        self.d1, self.d2, self.dr = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (y1, y2, rho))
        self.out = torch.zeros(self.n * FS_RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        torch.cuda.synchronize(dev)

    def call(self, ctx, L, st, s, q):
        return L.lcbi_gpu_binary_mag_noalloc(ctx.handle, C.byref(st), s, q, self.n, self.d1.data_ptr(),
                                             self.d2.data_ptr(), self.dr.data_ptr(), self.out.data_ptr())

    def results(self):
        from lcbinint_b200.api import FS_RESULT_DTYPE
        return self.out.cpu().numpy().view(FS_RESULT_DTYPE).copy()


def _noalloc(ctx, L, st, s, q, y1, y2, rho):
    d = _Device(ctx, y1, y2, rho)
    ctx.check(d.call(ctx, L, st, s, q), "lcbi_gpu_binary_mag_noalloc")
    return d.results()


def _same(a, b, skip=()):
    keep = np.ones(a.size, dtype=bool)
    keep[list(skip)] = False
    a, b = a[keep], b[keep]
    for f in ("magnification", "error_estimate"):
        x, y = a[f], b[f]
        assert np.array_equal(np.isnan(x), np.isnan(y)), f
        ok = ~np.isnan(x)
        assert np.array_equal(x[ok].view(np.int64), y[ok].view(np.int64)), \
            f"{f}: {np.sum(x[ok] != y[ok])} of {ok.sum()} differ"
    for f in ("method", "converged", "status", "seed_count"):
        assert np.array_equal(a[f], b[f]), f


@pytest.mark.parametrize("mode,c", [(1, 0.0), (2, 0.5), (4, 0.3)])
def test_noalloc_matches_workspace_entry_point_on_calls_in_a_row(mode, c):
    _lib_mod, L = _lib()
    ctx = _lib_mod.Context(0)
    try:
        st = _settings(mode, c)
        s1, q1 = 0.9, 1.0 / 0.05
        # 300 points: more than one 256-point pass of the fixed area.
        a1, a2, ar = _points(s1, q1, 300, seed=mode)
        ref_a = _workspace(ctx, L, st, s1, q1, a1, a2, ar)
        want = {1: {0, 1, 2}, 2: {0, 1, 3}, 4: {0, 1, 2, 3}}[mode]
        assert set(np.unique(ref_a["method"]).tolist()) >= want, np.unique(ref_a["method"])
        # Another lens model and other points in between: two rings whose
        # scans outgrow the first pass's share (second pass), then others.
        b1, b2, br = _ring_points([5e-3, 4e-3], 150, seed=10 + mode)
        ref_b = _workspace(ctx, L, st, *RING, b1, b2, br)
        assert (ref_b["method"][:2] >= 2).all() and (ref_b["status"][:2] == 0).all()
        first = _noalloc(ctx, L, st, s1, q1, a1, a2, ar)
        between = _noalloc(ctx, L, st, *RING, b1, b2, br)
        again = _noalloc(ctx, L, st, s1, q1, a1, a2, ar)
        _same(first, ref_a)
        _same(between, ref_b)
        _same(again, ref_a)
    finally:
        ctx.close()


def test_noalloc_rings_past_the_fixed_limits_get_status_18_and_19():
    _lib_mod, L = _lib()
    ctx = _lib_mod.Context(0)
    try:
        # Cartesian: a ring of rho = 2e-3 at 80 bins (source 1e-4 from the
        # lens) has about 85,000 rows in one seed's scans, past 65,536; polar:
        # rho = 1e-4 at 20 bins with the source 5e-5 from the lens (a whole
        # ring) visits about 272,000 segments, past 262,144 (the oracle's counts).
        for mode, rho_big, offset, status in ((1, 2e-3, 1e-4, 18), (2, 1e-4, 5e-5, 19)):
            st = _settings(mode, 0.4, bins=80 if mode == 1 else 20)
            y1, y2, rho = _ring_points([rho_big], 40, seed=mode, offset=offset)
            ref = _workspace(ctx, L, st, *RING, y1, y2, rho)
            assert ref["status"][0] == 0 and np.isfinite(ref["magnification"][0])
            got = _noalloc(ctx, L, st, *RING, y1, y2, rho)
            assert got["status"][0] == status, got["status"][0]
            assert np.isnan(got["magnification"][0])
            _same(got, ref, skip=[0])
    finally:
        ctx.close()


def test_noalloc_allocates_nothing_once_set_up():
    import torch
    _lib_mod, L = _lib()
    ctx = _lib_mod.Context(0)
    try:
        st = _settings(4, 0.3)
        y1, y2, rho = _ring_points([5e-3], 299, seed=3)
        d = _Device(ctx, y1, y2, rho)
        # The first call sets up (and loads the device code, whose fixed array
        # the driver reserves then); the next ones must not allocate.
        assert d.call(ctx, L, st, *RING) == _lib_mod.LCBI_OK
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(0)
        for _ in range(2):
            assert d.call(ctx, L, st, *RING) == _lib_mod.LCBI_OK
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(0)
        assert free1 == free0, (free0, free1)
        assert L.lcbi_gpu_workspace_bytes(ctx.handle) == 0
        assert d.results()["status"].max() == 0
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_the_fixed_area_and_refinement():
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
        st = _settings(1, 0.0, adaptive_source_bins=1, finite_source_reltol=1e-3)
        rc = L.lcbi_gpu_binary_mag_noalloc(ctx.handle, C.byref(st), 0.9, 20.0, 0, None, None, None, None)
        assert rc == _lib_mod.LCBI_UNSUPPORTED
    finally:
        ctx.close()
