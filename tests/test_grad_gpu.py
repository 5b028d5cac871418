"""GPU tests of the adjoint (lcbi_gpu_binary_mag_grad, lcbi_gpu_light_curves_grad
and the torch.autograd.Function over them).

Bars: point source and hexadecapole gradients are exact derivatives of the
forward's closed forms, so they match central finite differences of the
forward (relative step 1e-6) to 1e-5.  Inverse-ray gradients are the exact
gradients of a piecewise-linear approximation of the continuum magnification
(reported beside them), so they match its finite differences to 2e-3 (median,
scaled by the parameter's size; 1e-2 at the 75th percentile, the rest from
kinks of the piecewise-linear approximation and lattice squares joining the
visited set); that value agrees with the lattice forward to 2e-2,
and the source-position and rho gradients match finite differences of the
converged lattice forward (nbin 200, steps of 0.05 rho) to 1e-2 (median;
about 2e-3 measured, which the lattice forward's own differences set).
The rho gradient is not compared with differences of the continuum value:
its lattice spacing is rho / 50, so a relative change of rho of 1e-4 moves
lattice vertices a unit away from the origin by about one spacing, and those
differences measure the lattice's motion, not the magnification's.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _settings(mode=4, nbin=50, c=0.3, forced_ir=False):
    import lcbinint_b200 as lb
    st = lb.Options(nbin=nbin).fs_settings(lb.LimbDarkening.linear(c))
    st.finite_mode = mode
    if forced_ir:
        st.kinji_threshold = 1e18
        st.hex_threshold = 0.0
        st.adaptive_hex_threshold = 0.0
    return st


def _run(points_rows, settings_list):
    """rows: (s, q_core, y1, y2, rho, settings index) -> (results, grads (n, 8))."""
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, PS_EXACT, PS_ON_DEVICE, LcbiStructs
    rows = np.asarray(points_rows, dtype=np.float64)
    pts = np.zeros(len(rows), dtype=FS_POINT_DTYPE)
    pts["s"], pts["q"], pts["y1"], pts["y2"], pts["rho"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3], rows[:, 4]
    pts["settings"] = rows[:, 5].astype(np.int32)
    pts["flags"] = PS_EXACT | PS_ON_DEVICE
    res = np.zeros(len(rows), dtype=FS_RESULT_DTYPE)
    grads = np.zeros((len(rows), 8))
    st = (LcbiStructs.FsSettings * len(settings_list))(*settings_list)
    ctx = _lib.context(0)
    rc = ctx._L.lcbi_gpu_binary_mag_grad(ctx.handle, st, len(settings_list), None, 0, len(rows), pts.ctypes.data,
                                         res.ctypes.data, grads.ctypes.data, 0)
    ctx.check(rc, "lcbi_gpu_binary_mag_grad")
    return res, grads


def _near_caustic(n, seed, rho_range=(2e-3, 2e-2), spread=3.0):
    from oracle.oracle import Oracle
    rng = np.random.default_rng(seed)
    rows = []
    while len(rows) < n:
        s = float(np.exp(rng.uniform(np.log(0.6), np.log(1.6))))
        q = float(np.exp(rng.uniform(np.log(1e-3), 0.0)))
        rho = float(np.exp(rng.uniform(np.log(rho_range[0]), np.log(rho_range[1]))))
        br, _, _ = Oracle().caustic_cache(s, q, 256)
        pts = br.reshape(-1, 2)
        p = pts[rng.integers(len(pts))] + rng.normal(0.0, spread * rho, 2)
        rows.append([s, q, p[0], p[1], rho])
    return np.array(rows)


def _fd(rows, sidx, settings, k, h):
    """Central differences of (A, slot 6) in point parameter k (0 y1, 1 y2, 2 s, 3 q, 4 rho)."""
    col = {0: 2, 1: 3, 2: 0, 3: 1, 4: 4}[k]
    up = rows.copy()
    dn = rows.copy()
    up[:, col] += h
    dn[:, col] -= h
    ru, gu = _run(np.column_stack([up, sidx]), settings)
    rd, gd = _run(np.column_stack([dn, sidx]), settings)
    return ru, rd, gu, gd


def test_point_source_gradient_matches_finite_differences():
    rows = _near_caustic(200, seed=1, spread=20.0)
    st = [_settings(mode=0)]
    sidx = np.zeros(len(rows))
    res, g = _run(np.column_stack([rows, sidx]), st)
    assert (res["method"] == 0).all()
    A = res["magnification"]
    ok = A < 200.0
    for k in range(4):
        col = {0: 2, 1: 3, 2: 0, 3: 1}[k]
        h = 1e-6 * np.maximum(np.abs(rows[:, col]), 0.1)
        up, dn = rows.copy(), rows.copy()
        up[:, col] += h
        dn[:, col] -= h
        ru, _ = _run(np.column_stack([up, sidx]), st)
        rd, _ = _run(np.column_stack([dn, sidx]), st)
        fd = (ru["magnification"] - rd["magnification"]) / (2 * h)
        scale = np.abs(fd) + A / np.maximum(np.abs(rows[:, col]), 0.1)
        err = np.abs(g[:, k] - fd) / scale
        assert np.nanmax(err[ok]) < 1e-5, (k, np.nanmax(err[ok]))
    assert np.all(g[:, 4] == 0.0) and np.all(g[:, 5] == 0.0)


def test_hexadecapole_gradient_matches_finite_differences():
    rows = _near_caustic(300, seed=2, spread=6.0)
    st = [_settings(mode=4, c=0.4), _settings(mode=4, c=0.4 + 1e-6), _settings(mode=4, c=0.4 - 1e-6)]
    sidx = np.zeros(len(rows))
    res, g = _run(np.column_stack([rows, sidx]), st)
    hexm = res["method"] == 1
    assert hexm.sum() > 30
    A = res["magnification"]
    for k in range(5):
        col = {0: 2, 1: 3, 2: 0, 3: 1, 4: 4}[k]
        h = 1e-6 * np.abs(rows[:, col]) if k >= 2 else np.full(len(rows), 1e-6)
        ru, rd, _, _ = _fd(rows, sidx, st, k, h)
        same = hexm & (ru["method"] == 1) & (rd["method"] == 1)
        fd = (ru["magnification"] - rd["magnification"]) / (2 * h)
        size = np.abs(rows[:, col]) if k >= 2 else rows[:, 4]
        err = np.abs(g[:, k] - fd) * size / A
        assert np.nanmax(err[same]) < 1e-5, (k, np.nanmax(err[same]))
    ru, _ = _run(np.column_stack([rows, np.ones(len(rows))]), st)
    rd, _ = _run(np.column_stack([rows, np.full(len(rows), 2.0)]), st)
    same = hexm & (ru["method"] == 1) & (rd["method"] == 1)
    fd = (ru["magnification"] - rd["magnification"]) / 2e-6
    assert np.nanmax(np.abs(g[same, 5] - fd[same]) / A[same]) < 1e-5


@pytest.mark.parametrize("mode", [1, 2])
def test_inverse_ray_gradient_matches_its_continuum_value(mode):
    rows = _near_caustic(24, seed=3 + mode, rho_range=(3e-3, 1e-2), spread=1.0)
    c = 0.45
    st = [_settings(mode=mode, nbin=50, c=c, forced_ir=True), _settings(mode=mode, nbin=50, c=c + 1e-4, forced_ir=True),
          _settings(mode=mode, nbin=50, c=c - 1e-4, forced_ir=True)]
    sidx = np.zeros(len(rows))
    res, g = _run(np.column_stack([rows, sidx]), st)
    assert (res["method"] == mode + 1).all() and (res["status"] == 0).all()
    A = res["magnification"]
    Ac = g[:, 6]
    assert np.all(np.isfinite(g[:, :7]))
    # the continuum value the gradient differentiates agrees with the lattice forward
    assert np.max(np.abs(Ac / A - 1.0)) < 2e-2, np.max(np.abs(Ac / A - 1.0))
    rho = rows[:, 4]
    for k, h, size in ((0, 1e-4 * rho, rho), (1, 1e-4 * rho, rho), (2, 1e-6 * rows[:, 0], rows[:, 0]),
                       (3, 1e-6 * rows[:, 1], rows[:, 1])):
        _, _, gu, gd = _fd(rows, sidx, st, k, h)
        fd = (gu[:, 6] - gd[:, 6]) / (2 * h)
        err = np.abs(g[:, k] - fd) * size / Ac
        # The approximation is piecewise smooth (kinks where a lattice vertex
        # crosses a level), and a lattice cell that joins the visited set
        # adds a step of one square, so some points see finite-difference
        # error at any step; the bar is on the median and the 75th percentile.
        assert np.median(err) < 2e-3 and np.percentile(err, 75) < 1e-2, \
            (k, np.median(err), np.percentile(err, 75), np.max(err))
    _, gu = _run(np.column_stack([rows, np.ones(len(rows))]), st)
    _, gd = _run(np.column_stack([rows, np.full(len(rows), 2.0)]), st)
    fd = (gu[:, 6] - gd[:, 6]) / 2e-4
    err = np.abs(g[:, 5] - fd) / Ac
    assert np.median(err) < 1e-3 and np.max(err) < 1e-2, (np.median(err), np.max(err))


def test_inverse_ray_gradient_matches_converged_forward():
    rows = _near_caustic(12, seed=9, rho_range=(5e-3, 1e-2), spread=0.8)
    st = [_settings(mode=1, nbin=200, c=0.3, forced_ir=True)]
    sidx = np.zeros(len(rows))
    res, g = _run(np.column_stack([rows, sidx]), st)
    A = res["magnification"]
    rho = rows[:, 4]
    # The lattice forward moves in steps of its cells, so its differences need
    # steps of several cells; the bar is on the median over the points.
    for k, h, size in ((0, 0.05 * rho, rho), (1, 0.05 * rho, rho), (4, 0.05 * rho, rho)):
        ru, rd, _, _ = _fd(rows, sidx, st, k, h)
        fd = (ru["magnification"] - rd["magnification"]) / (2 * h)
        err = np.abs(g[:, k] - fd) * size / A
        assert np.median(err) < 1e-2, (k, np.median(err), np.max(err))


def test_light_curve_autograd_matches_finite_differences():
    import torch
    from lcbinint_b200.autograd import light_curve_magnification, light_curves_with_grad
    # Point-source and hexadecapole epochs: an event away from the caustic.
    P = np.array([[0.1, 20.0, 0.3, 0.7, 1.3, 0.01, 1e-3, 0.4], [-0.2, 15.0, 0.25, 2.0, 0.8, 0.05, 2e-3, 0.2]])
    T = np.linspace(-30.0, 30.0, 40)
    A, dA, method, status = light_curves_with_grad(P, T)
    assert (status == 0).all() and np.isin(method, [0, 1]).all()
    for j in range(8):
        h = 1e-6 * max(abs(P[0, j]), 1e-2)
        up, dn = P.copy(), P.copy()
        up[:, j] += h
        dn[:, j] -= h
        Au, _, mu, _ = light_curves_with_grad(up, T, with_grad=False)
        Ad, _, md, _ = light_curves_with_grad(dn, T, with_grad=False)
        same = (mu == method) & (md == method)
        fd = (Au - Ad) / (2 * h)
        err = np.abs(dA[..., j] - fd) * max(abs(P[0, j]), 1e-2) / A
        assert np.max(err[same]) < 1e-5, (j, np.max(err[same]))
    params = torch.tensor(P, requires_grad=True)
    At = light_curve_magnification(params, torch.tensor(T))
    assert np.array_equal(At.detach().numpy(), A)
    At.sum().backward()
    assert np.allclose(params.grad.numpy(), dA.sum(axis=1), rtol=1e-12, atol=0)


def test_device_resident_autograd_matches_the_host_arrays():
    """Times, magnifications and gradients as CUDA tensors
    (lcbi_gpu_light_curves_grad_device) give the host path's magnifications
    bit for bit, and torch.autograd runs through them on the device.  The
    inverse-ray gradients are sums that the gradient flood fill accumulates
    with FP64 atomic additions, whose order varies from run to run, so two
    runs agree to rounding of the summed magnitudes, not bit for bit."""
    import torch
    from lcbinint_b200.autograd import light_curve_magnification, light_curves_with_grad
    P = np.array([[0.0, 1.0, -0.01, 0.5, 0.95, 0.01, 5e-3, 0.5], [0.1, 20.0, 0.3, 0.7, 1.3, 0.01, 1e-3, 0.4],
                  [-0.2, 15.0, 0.05, 2.0, 0.8, 0.05, 2e-3, 0.2]])
    T = np.stack([np.linspace(-0.5, 0.5, 64), np.linspace(-30.0, 30.0, 64), np.linspace(-10.0, 10.0, 64)])
    A, dA, method, status = light_curves_with_grad(P, T)
    dev = torch.device("cuda", 0)
    params = torch.tensor(P, device=dev, requires_grad=True)
    times = torch.tensor(T, device=dev)
    At = light_curve_magnification(params, times)
    assert At.is_cuda
    a = At.detach().cpu().numpy()
    assert np.array_equal(np.isnan(a), np.isnan(A))
    ok = ~np.isnan(A)
    assert np.array_equal(a[ok].view(np.int64), A[ok].view(np.int64))
    (At * torch.arange(64, device=dev, dtype=torch.float64)).sum().backward()
    want = (dA * np.arange(64)[None, :, None]).sum(axis=1)
    got = params.grad.cpu().numpy()
    fin = np.isfinite(want)
    assert np.array_equal(np.isfinite(got), fin)
    # Rounding of a sum depends on its order: bound the difference by 1e-11 of
    # the magnitudes summed (the weighted per-epoch gradients), plus 1e-12
    # relative.
    scale = (np.abs(np.nan_to_num(dA, nan=0.0, posinf=0.0, neginf=0.0)) * np.arange(64)[None, :, None]).sum(axis=1)
    diff = np.abs(got[fin] - want[fin])
    assert (diff <= 1e-12 * np.abs(want[fin]) + 1e-11 * scale[fin]).all(), np.max(diff / (scale[fin] + 1e-300))


@pytest.mark.parametrize("mode", [1, 2])
def test_quadratic_limb_darkening_gradient_matches_its_continuum_value(mode):
    """Quadratic limb darkening (d != 0): finite gradients whose continuum value
    agrees with the lattice forward, and which match finite differences of that
    value in the source position, s and q at the linear law's bars, and
    finite differences of the converged lattice forward in rho."""
    import lcbinint_b200 as lb
    rows = _near_caustic(16, seed=13 + mode, rho_range=(3e-3, 1e-2), spread=1.0)
    st = lb.Options(nbin=50).fs_settings(lb.LimbDarkening.quadratic(0.3, 0.25))
    st.finite_mode = mode
    st.kinji_threshold = 1e18
    st.hex_threshold = 0.0
    st.adaptive_hex_threshold = 0.0
    sidx = np.zeros(len(rows))
    res, g = _run(np.column_stack([rows, sidx]), [st])
    assert (res["method"] == mode + 1).all() and (res["status"] == 0).all()
    assert np.all(np.isfinite(g[:, :7]))
    A = res["magnification"]
    Ac = g[:, 6]
    assert np.max(np.abs(Ac / A - 1.0)) < 2e-2, np.max(np.abs(Ac / A - 1.0))
    rho = rows[:, 4]
    # Thirteen contours (the linear law's seven and six for the quadratic
    # term) have more kinks than seven, so s and q take steps of 1e-8
    # relative, which straddle fewer of them.
    for k, h, size in ((0, 1e-4 * rho, rho), (1, 1e-4 * rho, rho), (2, 1e-8 * rows[:, 0], rows[:, 0]),
                       (3, 1e-8 * rows[:, 1], rows[:, 1])):
        _, _, gu, gd = _fd(rows, sidx, [st], k, h)
        fd = (gu[:, 6] - gd[:, 6]) / (2 * h)
        err = np.abs(g[:, k] - fd) * size / Ac
        assert np.median(err) < 2e-3 and np.percentile(err, 75) < 1e-2, \
            (k, np.median(err), np.percentile(err, 75), np.max(err), np.round(err, 4).tolist())
    if mode == 1:
        conv = lb.Options(nbin=200).fs_settings(lb.LimbDarkening.quadratic(0.3, 0.25))
        conv.finite_mode = 1
        conv.kinji_threshold = 1e18
        conv.hex_threshold = 0.0
        conv.adaptive_hex_threshold = 0.0
        h = 0.05 * rho
        ru, rd, _, _ = _fd(rows, sidx, [conv], 4, h)
        fd = (ru["magnification"] - rd["magnification"]) / (2 * h)
        err = np.abs(g[:, 4] - fd) * rho / A
        assert np.median(err) < 3e-2, (np.median(err), np.max(err))


def test_inverse_ray_gradient_converges_with_its_lattice():
    """The inverse-ray gradient is that of a piecewise-linear approximation on
    a lattice of rho / cells cells (lcbi_gpu_set_grad_resolution), whose error
    falls as the square of the cell: on near-caustic points the gradients and
    the continuum value at 48 and 96 cells per radius approach those at 192,
    the 96-cell ones closer (median over points and parameters)."""
    from lcbinint_b200 import _lib
    rows = _near_caustic(16, seed=21, rho_range=(3e-3, 1e-2), spread=1.0)
    st = [_settings(mode=1, nbin=50, c=0.4, forced_ir=True)]
    sidx = np.zeros(len(rows))
    ctx = _lib.context(0)
    out = {}
    try:
        for cells in (48, 96, 192):
            assert ctx._L.lcbi_gpu_set_grad_resolution(ctx.handle, cells) == 0
            res, g = _run(np.column_stack([rows, sidx]), st)
            assert (res["status"] == 0).all() and (res["method"] == 2).all()
            out[cells] = g
        assert ctx._L.lcbi_gpu_set_grad_resolution(ctx.handle, 4) != 0
    finally:
        ctx._L.lcbi_gpu_set_grad_resolution(ctx.handle, 48)
    ref = out[192]
    assert np.isfinite(ref[:, :7]).all()
    rho = rows[:, 4]
    # dA/d(y1, y2, rho) scaled by rho, dA/ds by s, relative to the magnification
    scale = np.column_stack([rho, rho, rows[:, 0], rho]) / ref[:, 6:7]
    cols = [0, 1, 2, 4]

    def dev(cells):
        d = np.abs(out[cells][:, cols] - ref[:, cols]) * scale
        return np.median(d), np.median(np.abs(out[cells][:, 6] / ref[:, 6] - 1.0))

    g48, a48 = dev(48)
    g96, a96 = dev(96)
    assert g96 < 0.6 * g48 and a96 < 0.6 * a48, (g48, g96, a48, a96)
