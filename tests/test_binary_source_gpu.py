"""Binary-source light curves: LightCurve(source="binary") blends two
single-source curves as (A1 + fr A2) / (1 + fr), the second source with its
own t0_2 and u0_2 (python/lcbinint_pybind.cpp:2331-2354).  Compared with the
reference's own module built from its sources (oracle/_ref) on the static
binary lens (the direct path) and under lens orbital motion (LensModel's
path), with finite sources and linear limb darkening.  Bar: bit-identical,
except polar inverse-ray points (an exact sum here, a running sum in the
reference: 1e-12 relative)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    """Bit for bit, except epochs integrated on the polar lattice (the auto
    grid takes it for |A_ps| >= 100): the same cells, summed exactly here and
    by a running sum in the reference, so they agree to 1e-12 relative."""
    a = np.asarray(a)
    b = np.asarray(b)
    eq = a.view(np.int64) == b.view(np.int64)
    rel = np.abs(a / b - 1.0)
    assert (eq | (rel <= 1e-12)).all(), f"{int((~eq).sum())} differ, max rel {np.nanmax(rel):.3e}"


@pytest.mark.parametrize("orbital", [False, True])
def test_binary_source_blend_matches_reference(orbital):
    import lcbinint_b200 as lb
    from oracle.oracle import import_reference_module
    ref = import_reference_module()
    if ref is None:
        pytest.skip("the reference module is not built (make -C oracle ref)")
    times = np.linspace(-0.6, 0.6, 160)
    p = dict(t0=0.0, tE=1.0, u0=-0.01, alpha=0.5, s=0.95, q=1e-2, rho=5e-3, t0_2=0.12, u0_2=0.05, flux_ratio=0.35)
    if orbital:
        p.update(g1=0.2, g2=-0.3, g3=0.05)
    mo = (lb.CIRCULAR, ref.CIRCULAR) if orbital else (lb.STATIC, ref.STATIC)
    for nbin in (20, 50):
        ours = lb.LightCurve(source="binary", options=lb.Options(nbin=nbin),
                             limb_darkening=lb.LimbDarkening.linear(0.5), orbital_motion_mode=mo[0])
        theirs = ref.LightCurve(source="binary", options=ref.Options(nbin=nbin),
                                limb_darkening=ref.LimbDarkening.linear(0.5), orbital_motion_mode=mo[1])
        A = ours(times, p)
        R = np.asarray(theirs(times, p))
        _same(A, R)
        # The blend itself, bit for bit, from this library's two single-source curves.
        one = lb.LightCurve(options=lb.Options(nbin=nbin), limb_darkening=lb.LimbDarkening.linear(0.5),
                            orbital_motion_mode=mo[0])
        p2 = dict(p, u0=p["u0_2"], t0=p["t0_2"])
        fr = p["flux_ratio"]
        blend = (one(times, p) + fr * one(times, p2)) * (1.0 / (1.0 + fr))
        assert np.array_equal(A.view(np.int64), blend.view(np.int64))
        # The blend really mixes two different curves.
        single = lb.LightCurve(options=lb.Options(nbin=nbin), limb_darkening=lb.LimbDarkening.linear(0.5),
                               orbital_motion_mode=mo[0])
        assert not np.allclose(A, single(times, p))
    # flux_ratio 0 leaves the first source's curve.
    q0 = dict(p, flux_ratio=0.0)
    ours = lb.LightCurve(source="binary", limb_darkening=lb.LimbDarkening.linear(0.5), orbital_motion_mode=mo[0])
    single = lb.LightCurve(limb_darkening=lb.LimbDarkening.linear(0.5), orbital_motion_mode=mo[0])
    _same(ours(times, q0), single(times, q0))
