"""Adaptive local refinement (finite_source_tol / finite_source_reltol with
adaptive_source_bins; fixed_inverse_ray_binary,
src/lcbinint/magnification/finite_source_magnifier.cpp:3074-3294) against the
reference built from its sources (oracle/_ref): the tape of boundary cells
recorded by the Cartesian scan, the priority-queue refinement, the
refined magnification, its error estimate, the convergence flag and the
refinement level."""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

pytestmark = pytest.mark.gpu


def _reference():
    from oracle.oracle import Reference, have_reference
    if not have_reference():
        pytest.skip("oracle/_ref not built")
    return Reference()


@pytest.mark.parametrize("tol,reltol,ld", [(0.0, 1e-4, 0.0), (0.0, 3e-4, 0.5), (1e-3, 0.0, 0.3)])
def test_refined_cartesian_points_match_reference(tol, reltol, ld):
    import bench
    import lcbinint_b200 as lb
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, LcbiStructs, PS_EXACT
    from oracle.oracle import default_settings
    ref = _reference()
    rows = bench.fs_batch_workload(seed=1)
    rows = rows[rows[:, 6] == 1]  # the Cartesian points
    rows = rows[np.random.default_rng(4).permutation(len(rows))[:48]]
    ctx = _lib.Context(0)
    mismatches = []
    refined = 0
    for r in rows:
        s, q, x, y, rho = r[0], r[1], r[2], r[3], r[4]
        nbin = int(r[7])
        kw = dict(source_bins=nbin, finite_mode=1, kinji_threshold=1e18, hex_threshold=0.0, adaptive_hex_threshold=0.0,
                  limb_darkening_c=ld, adaptive_source_bins=1, max_source_bins=400, finite_source_tol=tol,
                  finite_source_reltol=reltol)
        a_ps = float(ref.binary_mag0(s, q, x, y)[0][0])
        want = ref.binary_mag(default_settings(**kw), s, q, x, y, rho, a_ps, True)
        st = LcbiStructs.FsSettings(source_bins=nbin, caustic_bins=1400, grid_ratio=4.0, polar_source_bins=0,
                                    polar_grid_ratio=0.0, finite_mode=1, kinji_threshold=1e18, hex_threshold=0.0,
                                    adaptive_hex_threshold=0.0, limb_darkening_c=ld, limb_darkening_d=0.0,
                                    adaptive_source_bins=1, max_source_bins=400, finite_source_tol=tol,
                                    finite_source_reltol=reltol)
        pts = np.zeros(1, dtype=FS_POINT_DTYPE)
        pts[0] = (s, q, x, y, rho, a_ps, 0, 0, PS_EXACT, 0)
        res = np.zeros(1, dtype=FS_RESULT_DTYPE)
        ctx.check(ctx._L.lcbi_gpu_binary_mag(ctx.handle, C.byref(st), 1, None, 0, 1, pts.ctypes.data,
                                             res.ctypes.data, 0), "lcbi_gpu_binary_mag")
        got = res[0]
        refined += want["level"] > 0
        ok = (got["status"] == 0 and got["method"] == want["method"] and
              np.float64(got["magnification"]).view(np.int64) == np.float64(want["A"]).view(np.int64) and
              np.float64(got["error_estimate"]).view(np.int64) == np.float64(want["err"]).view(np.int64) and
              bool(got["converged"]) == want["converged"])
        if not ok:
            mismatches.append((r.tolist(), dict(got=got.tolist(), want=want)))
    assert not mismatches, mismatches[:3]
    assert refined > 0  # the refinement loop ran on some points


def test_refinement_level_through_the_c_abi():
    """lcbi_magnification_array with adaptive options: every result field,
    the refinement level included, as the compiled reference's."""
    import test_capi_compat as TC
    from lcbinint_b200 import api
    import lcbinint_b200 as lb
    ours, theirs = TC._ours(), TC._reference()
    p = api.binary_c_params([dict(t0=0.0, tE=1.0, u0=-0.01, alpha=0.5, s=0.95, q=1e-2, rho=5e-3)],
                            lb.LimbDarkening.linear(0.5))
    P = TC.Params.from_buffer_copy(p.tobytes())
    o = ours.lcbi_default_options()
    o.adaptive_source_bins = 1
    o.finite_source_reltol = 1e-4
    o.mode = 1
    o.source_bins = 40
    times = np.ascontiguousarray(np.linspace(-0.5, 0.5, 120))
    a = (TC.Result * len(times))()
    b = (TC.Result * len(times))()
    sa = ours.lcbi_magnification_array(times.ctypes.data, len(times), C.byref(P), C.byref(o), a)
    sb = theirs.lcbi_magnification_array(times.ctypes.data, len(times), C.byref(P), C.byref(o), b)
    assert sa == sb
    fa, fb = TC._fields(a), TC._fields(b)
    assert (fb["finite_source_refinement_level"] > 0).any()
    for f in fa:
        x, y = fa[f], fb[f]
        if x.dtype.kind == "f":
            assert np.array_equal(np.isnan(x), np.isnan(y)), f
            ok = ~np.isnan(x)
            assert np.array_equal(x[ok].view(np.int64), y[ok].view(np.int64)), (f, np.nanmax(np.abs(x / y - 1.0)))
        else:
            assert np.array_equal(x, y), f
