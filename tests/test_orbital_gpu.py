"""Lens orbital motion and the original / centre-of-mass conventions through
lcbinint_b200.LightCurve, against the reference's own Python module built from
its sources (oracle/_ref).

The reference routes these light curves two ways: a parameter dictionary goes
through LensModel (python/lcbinint_pybind.cpp:2325-2358 ->
src/lcbinint/model/lens_model.cpp:83-236) and keyword parameters through the
module's dynamic path (python/lcbinint_pybind.cpp:1364-1385, 1958-2060).
Both are checked value for value: the source positions, orbits and every
magnification method but the polar sum are bit-exact, so the bar is equality
(1e-12 relative for polar points).
"""
import numpy as np
import pytest

import lcbinint_b200 as lb
from lcbinint_b200 import api

pytestmark = pytest.mark.gpu


def _ref():
    from oracle.oracle import have_reference, import_reference_module
    if not have_reference():
        pytest.skip("oracle/_ref not built")
    return import_reference_module()


def _model(rng, mode):
    p = dict(t0=float(rng.uniform(-5, 5)), tE=float(rng.uniform(10.0, 40.0)), u0=float(rng.uniform(-0.15, 0.15)),
             alpha=float(rng.uniform(0, 2 * np.pi)), s=float(np.exp(rng.uniform(np.log(0.5), np.log(2.0)))),
             q=float(np.exp(rng.uniform(np.log(1e-3), 0.0))), rho=float(np.exp(rng.uniform(np.log(5e-4), np.log(5e-3)))))
    if mode != api.STATIC:
        p.update(g1=float(rng.uniform(-1, 1)) / 365.25, g2=float(rng.uniform(-1, 1)) / 365.25,
                 g3=float(rng.uniform(0.0, 0.5)) / 365.25)
    if mode == api.KEPLER:
        p.update(lom_szs=float(rng.uniform(-0.5, 0.5)), lom_ar=float(rng.uniform(1.0, 2.0)))
    return p


def _pair(ref, mode, coordinates, c):
    ours = lb.LightCurve(options=lb.Options(coordinates=coordinates), limb_darkening=lb.LimbDarkening.linear(c),
                         orbital_motion_mode=mode)
    theirs = ref.LightCurve(options=ref.Options(coordinates=coordinates), limb_darkening=ref.LimbDarkening.linear(c),
                            orbital_motion_mode=[ref.STATIC, ref.CIRCULAR, ref.KEPLER][mode])
    return ours, theirs


def _compare(a, b):
    """Bit-identical, except that polar inverse-ray points may differ in the
    last bits: their sum is exact here (128-bit fixed point) and a running
    FP64 sum in the reference (1e-12 relative bounds the difference)."""
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape
    same = a.view(np.int64) == b.view(np.int64)
    rel = np.abs(a / b - 1.0)
    assert (same | (rel <= 1e-12)).all(), (int((~same).sum()), float(np.max(rel)))
    assert same.mean() >= 0.9


@pytest.mark.parametrize("mode", [api.CIRCULAR, api.KEPLER])
@pytest.mark.parametrize("coordinates", ["vbm", "lcbinint", "center_of_mass"])
def test_orbital_light_curve_dictionary_route(mode, coordinates):
    ref = _ref()
    rng = np.random.default_rng(300 + mode)
    times = np.linspace(-60.0, 60.0, 150)
    for _ in range(2):
        p = _model(rng, mode)
        ours, theirs = _pair(ref, mode, coordinates, 0.45)
        _compare(ours(times, p), theirs(times, p))


@pytest.mark.parametrize("mode", [api.CIRCULAR, api.KEPLER])
@pytest.mark.parametrize("coordinates", ["vbm", "lcbinint"])
def test_orbital_light_curve_keyword_route(mode, coordinates):
    ref = _ref()
    rng = np.random.default_rng(310 + mode)
    times = np.linspace(-60.0, 60.0, 150)
    p = _model(rng, mode)
    ours, theirs = _pair(ref, mode, coordinates, 0.3)
    _compare(ours(times, **p), theirs(times, **p))


@pytest.mark.parametrize("coordinates", ["lcbinint", "center_of_mass"])
def test_static_light_curve_in_other_conventions(coordinates):
    """The static binary outside VBM coordinates also leaves the direct path."""
    ref = _ref()
    rng = np.random.default_rng(320)
    times = np.linspace(-40.0, 40.0, 120)
    p = _model(rng, api.STATIC)
    p["s"] = 1.4  # wide enough for the wide-binary offset of the original convention
    ours, theirs = _pair(ref, api.STATIC, coordinates, 0.5)
    _compare(ours(times, p), theirs(times, p))
    _compare(ours(times, **p), theirs(times, **p))


def test_batched_sets_match_single_calls():
    """Many parameter sets in one lcbi_gpu_magnification_arrays pass give the
    records lcbi_magnification_array gives one set at a time."""
    rng = np.random.default_rng(330)
    dicts, times = [], []
    for m in range(6):
        mode = [api.STATIC, api.CIRCULAR, api.KEPLER][m % 3]
        p = _model(rng, mode)
        p["rho"] = 0.0 if m == 4 else p["rho"]
        dicts.append((p, mode))
        times.append(np.linspace(-50.0, 50.0, 40 + 7 * m))
    cps = np.concatenate([api.binary_c_params([p], lb.LimbDarkening.linear(0.2 * (m % 3)), orbital_motion_mode=mode)
                          for m, (p, mode) in enumerate(dicts)])
    opts = lb.Options(coordinates="lcbinint")
    batched, status = api.magnification_arrays(times, cps, opts)
    assert (status == 0).all()
    for m in range(len(dicts)):
        (single,), st = api.magnification_arrays([times[m]], cps[m:m + 1], opts)
        assert st[0] == 0
        assert batched[m].tobytes() == single.tobytes()


def test_status_per_set():
    """Per-set statuses as lcbi_magnification_array reports them: an invalid
    set, an unsupported one (a triple lens) and a good one in one batch."""
    rng = np.random.default_rng(340)
    good = _model(rng, api.CIRCULAR)
    cps = api.binary_c_params([good, good, good], orbital_motion_mode=api.CIRCULAR)
    cps[0]["tE"] = 0.0
    cps[1]["q2"] = 0.2
    times = [np.linspace(-10, 10, 5)] * 3
    res, status = api.magnification_arrays(times, cps)
    assert list(status) == [1, 3, 0]
    assert np.isnan(res[1]["magnification"][0])
    assert np.isfinite(res[2]["magnification"]).all()
