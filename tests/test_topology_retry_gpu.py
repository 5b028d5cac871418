"""The topology retry of fixed_inverse_ray_binary
(src/lcbinint/magnification/finite_source_magnifier.cpp:3168-3196): with
adaptive_source_bins set, a Cartesian point scanned at fewer than 50 bins
whose scan shows at least 16 seeds, 100 overlaps, 1,000 gap repairs and a
1,000-cell jump (needs_global_topology_retry, :1108-1121) is scanned again at
min(max_source_bins, max(50, 2 nbin)) bins, and the rescan's magnification,
diagnostics and boundary tape replace the first one's (refinement level 1,
then the local refinement on top when a tolerance is set).

The points are caustic crossings of planetary and resonant lenses found by a
seeded search with the reference's own scan diagnostics (every one of them
meets the trigger).  Each is compared with the reference built from its
sources (oracle/_ref), forced to inverse ray, in magnification, error
estimate, convergence flag and refinement level, bit for bit, with no
tolerance (the retry alone), a loose one (the retry meets it) and a tight one
(the local refinement splits cells after the retry), and with limb
darkening."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (s, q, x, y, rho, nbin): s, q in the core convention (q > 1 inverted).
POINTS = [
    (1.3869610818437774, 971.6996997020298, 0.0006145515061301674, -0.00014431688280591904, 0.0013788701516018053, 48),
    (1.7068649343568325, 120.39202941931613, 0.01164880394384615, -0.0006571265194235405, 0.0013331339185451998, 29),
    (1.5953611364741773, 4.059040480917747, 0.22107586638666532, 0.07231564330547084, 0.00220737780549818, 45),
    (1.024939914945014, 1018.9810663027682, 0.0013267133367403476, -0.0011884469038379298, 0.0018406206447359106, 20),
    (0.7538529354465361, 135.09736722047973, 0.0026166950510314556, -0.002611235176313911, 0.006677143693921839, 40),
    (0.9269117035965997, 1969.9083516895982, 0.002476388418698029, -0.0023483988598067243, 0.0031332052440187774, 44),
    (0.6691094674428328, 196.04900982861705, 0.0009687733670465757, 0.0032962456585520807, 0.0013031798505122338, 36),
    (0.7488776125567439, 201.55399691898478, 0.00034452841520867016, -0.0012537674427675867, 0.0043269855769974, 49),
    (0.985778328068777, 1288.9844286529735, 0.000713153816622153, 0.00024272606454815506, 0.00267718343584564, 44),
    (1.7395216436916097, 107.68528813886101, 0.01208397872795306, 0.001801281131875678, 0.0012763076013296414, 44),
    (0.8243057421614738, 1109.7995044459597, 0.00019851992612887764, 0.0002536380536864863, 0.0011622662148413282, 33),
    (0.5951586462110419, 976.0963073616931, 0.0001350991488234655, -0.0001917291223052943, 0.0011635721146708907, 30),
]


@pytest.mark.parametrize("reltol,ld", [(0.0, 0.0), (1e-3, 0.4), (2e-5, 0.0), (2e-5, 0.6)])
def test_topology_retry_matches_reference(reltol, ld, ref_lib):
    from lcbinint_b200 import _lib
    from lcbinint_b200.api import FS_POINT_DTYPE, FS_RESULT_DTYPE, PS_EXACT, LcbiStructs
    from oracle.oracle import default_settings
    kw = dict(finite_mode=1, kinji_threshold=1e18, hex_threshold=0.0, adaptive_hex_threshold=0.0,
              limb_darkening_c=ld, adaptive_source_bins=1, max_source_bins=400, finite_source_tol=0.0,
              finite_source_reltol=reltol)
    settings = []
    index = {}
    pts = np.zeros(len(POINTS), dtype=FS_POINT_DTYPE)
    want = []
    for i, (s, q, x, y, rho, nbin) in enumerate(POINTS):
        if nbin not in index:
            index[nbin] = len(settings)
            settings.append(LcbiStructs.FsSettings(
                source_bins=nbin, caustic_bins=1400, grid_ratio=4.0, polar_source_bins=0, polar_grid_ratio=0.0,
                limb_darkening_d=0.0, **kw))
        a_ps = float(ref_lib.binary_mag0(s, q, x, y)[0][0])
        pts[i] = (s, q, x, y, rho, a_ps, index[nbin], 0, PS_EXACT, 0)
        want.append(ref_lib.binary_mag(default_settings(source_bins=nbin, **kw), s, q, x, y, rho, a_ps, True))
    st = (LcbiStructs.FsSettings * len(settings))(*settings)
    ctx = _lib.Context(0)
    try:
        res = np.zeros(len(pts), dtype=FS_RESULT_DTYPE)
        ctx.check(ctx._L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings), None, 0, len(pts), pts.ctypes.data,
                                             res.ctypes.data, 0), "lcbi_gpu_binary_mag")
        levels = np.zeros(len(pts), dtype=np.int32)
        ctx.check(ctx._L.lcbi_gpu_last_refinement_levels(ctx.handle, len(pts), levels.ctypes.data),
                  "lcbi_gpu_last_refinement_levels")
    finally:
        ctx.close()
    bad = []
    for i, w in enumerate(want):
        g = res[i]
        same = (g["status"] == 0 and g["method"] == w["method"] == 2 and
                np.float64(g["magnification"]).view(np.int64) == np.float64(w["A"]).view(np.int64) and
                np.float64(g["error_estimate"]).view(np.int64) == np.float64(w["err"]).view(np.int64) and
                bool(g["converged"]) == w["converged"] and levels[i] == w["level"])
        if not same:
            bad.append((i, g.tolist(), int(levels[i]), w))
    assert not bad, bad[:3]
    lv = np.array([w["level"] for w in want])
    assert (lv >= 1).all()  # every point was scanned again
    if reltol == 2e-5:
        assert (lv > 1).any()  # and the local refinement split cells after the retry


def test_topology_retry_through_the_c_abi(ref_lib):
    """lcbi_magnification_array with adaptive options on a planetary caustic
    crossing at 24 bins: every result field, the refinement level included,
    as the compiled reference's (no point gets the old status 21)."""
    import test_capi_compat as TC
    import lcbinint_b200 as lb
    from lcbinint_b200 import api
    ours, theirs = TC._ours(), TC._reference()
    p = api.binary_c_params([dict(t0=0.0, tE=1.0, u0=0.0015, alpha=0.3, s=1.02, q=1.0 / 1018.98, rho=1.8e-3)],
                            lb.LimbDarkening.linear(0.5))
    P = TC.Params.from_buffer_copy(p.tobytes())
    o = ours.lcbi_default_options()
    o.adaptive_source_bins = 1
    o.finite_source_reltol = 1e-3
    o.mode = 1
    o.source_bins = 24
    times = np.ascontiguousarray(np.linspace(-0.01, 0.01, 64))
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
