"""GPU parity tests of the finite-source path through the C ABI.

Bar: bit-exact against the reference (oracle/_ref when present, else the
oracle restatement, which is bit-exact against it), on forced inverse-ray
points (Cartesian and polar, uniform and limb-darkened), on the full decision
tree, and on the README light curve.  The all-FP64 finite-source tolerance
stated for this path is 1e-6 relative; bit-exactness is checked first and the
tolerance is the acceptance bound reported on failure.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FS_REL_TOL = 1e-6


def _checker():
    from oracle.oracle import Oracle, Reference, have_reference
    return Reference() if have_reference() else Oracle()


def _near_caustic_cases(n_models, per_model, seed):
    from oracle.oracle import Oracle
    orc = Oracle()
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(n_models):
        s = float(np.exp(rng.uniform(np.log(0.3), np.log(3.0))))
        q = float(np.exp(rng.uniform(np.log(1e-4), 0.0)))
        rho = float(np.exp(rng.uniform(np.log(1e-3), np.log(3e-2))))
        c = float(rng.uniform(0.0, 0.8))
        br, _, _ = orc.caustic_cache(s, 1.0 / q, 256)
        pts = br.reshape(-1, 2)
        for _ in range(per_model):
            p = pts[rng.integers(len(pts))] + rng.normal(0.0, rho, 2)
            rows.append((s, 1.0 / q, p[0], p[1], rho, c))
    return np.array(rows)


def _report(A, R):
    rel = np.abs(A / R - 1.0)
    return f"max rel {np.nanmax(rel):.3e}, bit-exact {np.sum(A.view(np.int64) == R.view(np.int64))}/{A.size}"


def test_inverse_ray_golden_fixture(golden):
    import lcbinint_b200 as lb
    g = golden("inverse_ray.npz")
    for mode in (1, 2):
        sel = g["mode"] == mode
        grid = "cartesian" if mode == 1 else "polar"
        out = []
        for k in np.nonzero(sel)[0]:
            opt = lb.Options(inverse_ray_grid=grid, nbin=int(g["nbin"][k]))
            out.append(lb.binary_inverse_ray(g["s"][k], g["q"][k], g["x"][k], g["y"][k], g["rho"][k],
                                             lb.LimbDarkening.linear(g["ld_c"][k]), opt))
        A = np.array(out)
        R = g["A"][sel]
        assert np.allclose(A, R, rtol=FS_REL_TOL, atol=0), _report(A, R)


@pytest.mark.parametrize("grid", ["cartesian", "polar", "auto"])
def test_inverse_ray_batch_vs_reference(grid):
    import lcbinint_b200 as lb
    from oracle.oracle import default_settings
    ref = _checker()
    cases = _near_caustic_cases(12, 6, seed={"cartesian": 1, "polar": 2, "auto": 3}[grid])
    mode = {"cartesian": 1, "polar": 2, "auto": 4}[grid]
    for nbin in (20, 40):
        A_all = []
        R_all = []
        M_all = []
        for c in np.unique(cases[:, 5]):
            sel = cases[:, 5] == c
            s, q, x, y, rho = (cases[sel, i] for i in range(5))
            opt = lb.Options(inverse_ray_grid=grid, nbin=nbin)
            A, m, st = lb.binary_inverse_ray_batch(s, q, x, y, rho, lb.LimbDarkening.linear(c), opt,
                                                   return_method=True)
            R, rm = ref.inverse_ray(default_settings(source_bins=nbin, finite_mode=mode, limb_darkening_c=c),
                                    s, q, x, y, rho)
            assert np.array_equal(m, rm)
            assert (st == 0).all()
            A_all.append(A)
            R_all.append(R)
            M_all.append(m)
        A = np.concatenate(A_all)
        R = np.concatenate(R_all)
        M = np.concatenate(M_all)
        assert np.allclose(A, R, rtol=FS_REL_TOL, atol=0), _report(A, R)
        # Cartesian: the same cells visited in the same order -> bit-identical.
        cart = M == 2
        assert np.array_equal(A[cart].view(np.int64), R[cart].view(np.int64)), _report(A[cart], R[cart])
        # Polar: the same cell set, summed exactly -> equal up to the reference's own rounding.
        pol = M == 3
        assert np.allclose(A[pol], R[pol], rtol=1e-12, atol=0), _report(A[pol], R[pol])


def test_decision_tree_vs_reference():
    """Default thresholds (point source / hexadecapole / inverse ray) on points near and away
    from caustics; methods and magnifications must agree."""
    import lcbinint_b200 as lb
    from lcbinint_b200.api import FS_POINT_DTYPE, PS_EXACT, PS_ON_DEVICE
    from oracle.oracle import default_settings
    ref = _checker()
    cases = _near_caustic_cases(10, 8, seed=9)
    rng = np.random.default_rng(4)
    far = cases.copy()
    far[:, 2:4] += rng.normal(0.0, 0.05, (len(far), 2))
    allc = np.concatenate([cases, far])
    opt = lb.Options(nbin=30)
    sts = []
    pts = np.zeros(len(allc), dtype=FS_POINT_DTYPE)
    cvals = sorted(set(allc[:, 5]))
    for c in cvals:
        sts.append(opt.fs_settings(lb.LimbDarkening.linear(c)))
    for i, r in enumerate(allc):
        pts[i] = (r[0], r[1], r[2], r[3], r[4], 0.0, cvals.index(r[5]), 0, PS_EXACT | PS_ON_DEVICE, 0)
    res = lb.binary_mag(pts, sts)
    for i, r in enumerate(allc):
        a_ps = ref.binary_mag0([r[0]], [r[1]], [r[2]], [r[3]])[0][0]
        want = ref.binary_mag(default_settings(source_bins=30, finite_mode=4, limb_darkening_c=r[5]),
                              r[0], r[1], r[2], r[3], r[4], a_ps, True)
        assert res["method"][i] == want["method"], (i, res[i], want)
        assert res["status"][i] == 0
        assert abs(res["magnification"][i] / want["A"] - 1.0) <= FS_REL_TOL, (i, res[i], want)


def test_readme_light_curve(golden):
    import lcbinint_b200 as lb
    g = golden("light_curve_readme.npz")
    p = dict(t0=0.0, tE=1.0, u0=-0.01, alpha=0.5, s=0.95, q=1e-2, rho=5e-3)
    for name, grid in (("auto", "auto"), ("cartesian", "cartesian")):
        lc = lb.LightCurve(options=lb.Options(coordinates="vbm", nbin=50, inverse_ray_grid=grid),
                           limb_darkening=lb.LimbDarkening.linear(0.5))
        A = lc(g["times"], p)
        R = g[f"A_{name}"]
        assert np.allclose(A, R, rtol=FS_REL_TOL, atol=0), _report(A, R)
        info = lc.info(g["times"], p)
        assert np.array_equal(np.array(info.finite_source_methods), g[f"method_{name}"])


def test_zero_radius_and_far_sources():
    import lcbinint_b200 as lb
    lc = lb.LightCurve(options=lb.Options(nbin=20))
    t = np.linspace(-1, 1, 50)
    A0 = lc(t, dict(t0=0.0, tE=1.0, u0=0.5, alpha=0.3, s=1.2, q=0.3, rho=0.0))
    x = (t - 0.0) * (1.0 / 1.0) * np.cos(0.3) - 0.5 * np.sin(0.3)
    y = (t - 0.0) * (1.0 / 1.0) * np.sin(0.3) + 0.5 * np.cos(0.3)
    B = lb.binary_mag0_batch(1.2, 1.0 / 0.3, x, y)
    assert np.array_equal(A0, B)


@pytest.mark.parametrize("grid", ["cartesian", "polar"])
def test_block_pass_matches_warp_pass(grid):
    """Every scan implementation gives bit-for-bit the same results, and they
    match the reference: the first pass (Cartesian one warp per point; polar
    tile-parallel flood fill, or one warp per point) and the second pass (one
    block per point, here for every point: cell budget 1)."""
    import lcbinint_b200 as lb
    from lcbinint_b200 import _lib
    from oracle.oracle import default_settings
    ref = _checker()
    ctx = _lib.context(0)
    cases = _near_caustic_cases(8, 5, seed={"cartesian": 31, "polar": 32}[grid])
    mode = {"cartesian": 1, "polar": 2}[grid]
    nbin = 45
    out = {}
    runs = [(1 << 19, 1), (1 << 19, 0), (1, 0)]  # (cell budget, polar tiles)
    try:
        for budget, tiles in runs:
            assert ctx._L.lcbi_gpu_set_cell_budget(ctx.handle, budget) == 0
            assert ctx._L.lcbi_gpu_set_polar_tiles(ctx.handle, tiles) == 0
            A_all, M_all, S_all = [], [], []
            for c in np.unique(cases[:, 5]):
                sel = cases[:, 5] == c
                s, q, x, y, rho = (cases[sel, i] for i in range(5))
                A, m, st = lb.binary_inverse_ray_batch(s, q, x, y, rho, lb.LimbDarkening.linear(c),
                                                       lb.Options(inverse_ray_grid=grid, nbin=nbin),
                                                       return_method=True)
                A_all.append(A)
                M_all.append(m)
                S_all.append(st)
            out[(budget, tiles)] = (np.concatenate(A_all), np.concatenate(M_all), np.concatenate(S_all))
    finally:
        ctx._L.lcbi_gpu_set_cell_budget(ctx.handle, 1 << 19)
        ctx._L.lcbi_gpu_set_polar_tiles(ctx.handle, 1)
    A0, M0, S0 = out[runs[0]]
    assert (S0 == 0).all()
    for key in runs[1:]:
        A1, M1, S1 = out[key]
        assert (S1 == 0).all()
        assert np.array_equal(M0, M1)
        assert np.array_equal(A0.view(np.int64), A1.view(np.int64)), (key, _report(A1, A0))
    R_all = []
    for c in np.unique(cases[:, 5]):
        sel = cases[:, 5] == c
        s, q, x, y, rho = (cases[sel, i] for i in range(5))
        R, _ = ref.inverse_ray(default_settings(source_bins=nbin, finite_mode=mode, limb_darkening_c=c),
                               s, q, x, y, rho)
        R_all.append(R)
    R = np.concatenate(R_all)
    if grid == "cartesian":
        assert np.array_equal(A1.view(np.int64), R.view(np.int64)), _report(A1, R)
    else:
        assert np.allclose(A1, R, rtol=1e-12, atol=0), _report(A1, R)
