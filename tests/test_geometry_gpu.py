"""LightCurve.caustics / critical_curves and the orbital-motion functions,
value for value against the reference's own Python module (oracle/_ref):
python/lcbinint_pybind.cpp:1525-1561, 1882-1926 (geometry branches) and
:3896-3925 (circular_orbital_motion, kepler_orbital_motion)."""
import math

import numpy as np
import pytest

import lcbinint_b200 as lb

pytestmark = pytest.mark.gpu


def _ref():
    from oracle.oracle import have_reference, import_reference_module
    if not have_reference():
        pytest.skip("oracle/_ref not built")
    return import_reference_module()


def _same(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.int64), b.view(np.int64)), float(np.nanmax(np.abs(a - b)))


@pytest.mark.parametrize("coordinates", ["vbm", "lcbinint"])
@pytest.mark.parametrize("s,q,n", [(1.0, 1.0, 200), (0.7, 1e-3, 1400), (2.2, 3e-4, 500), (1.05, 0.2, 64), (0.4, 0.05, 8)])
def test_static_geometry_matches_reference(coordinates, s, q, n):
    ref = _ref()
    ours = lb.LightCurve(options=lb.Options(coordinates=coordinates))
    theirs = ref.LightCurve(options=ref.Options(coordinates=coordinates))
    for name in ("caustics", "critical_curves"):
        a = getattr(ours, name)(s=s, q=q, n_points=n)
        b = getattr(theirs, name)(s=s, q=q, n_points=n)
        _same(a.x, b.x)
        _same(a.y, b.y)
    a = ours.caustics({"s": s, "q": q})
    b = theirs.caustics({"s": s, "q": q})
    _same(a.x, b.x)
    _same(a.y, b.y)


@pytest.mark.parametrize("mode", [lb.CIRCULAR, lb.KEPLER])
def test_orbital_geometry_matches_reference(mode):
    ref = _ref()
    kw = dict(s=1.1, q=4e-3, n_points=300, time=37.0, t0=2.0, tE=25.0, u0=0.1, alpha=0.8,
              g1=0.4 / 365.25, g2=-0.3 / 365.25, g3=0.1 / 365.25, lom_szs=0.2, lom_ar=1.4)
    ours = lb.LightCurve(orbital_motion_mode=mode)
    theirs = ref.LightCurve(orbital_motion_mode=[ref.STATIC, ref.CIRCULAR, ref.KEPLER][mode])
    for name in ("caustics", "critical_curves"):
        a = getattr(ours, name)(**kw)
        b = getattr(theirs, name)(**kw)
        _same(a.x, b.x)
        _same(a.y, b.y)


def test_geometry_rejects_too_few_points():
    with pytest.raises(ValueError):
        lb.LightCurve().caustics(s=1.0, q=1.0, n_points=7)


def test_orbital_motion_functions_match_reference():
    ref = _ref()
    rng = np.random.default_rng(5)
    for _ in range(50):
        t, s, a = float(rng.uniform(-300, 300)), float(rng.uniform(0.3, 3)), float(rng.uniform(0, 2 * math.pi))
        g = [float(v) for v in rng.uniform(-1, 1, 3) / 365.25]
        tref = float(rng.uniform(-10, 10))
        _same(lb.circular_orbital_motion(t, s, a, *g, tref), ref.circular_orbital_motion(t, s, a, *g, tref))
        szs, ar = float(rng.uniform(-0.5, 0.5)), float(rng.uniform(1.0, 2.0))
        _same(lb.kepler_orbital_motion(t, s, a, *g, szs, ar, tref), ref.kepler_orbital_motion(t, s, a, *g, szs, ar, tref))
