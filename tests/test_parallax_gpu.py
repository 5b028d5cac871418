"""Annual and terrestrial parallax and xallarap (src/lcbinint/model/trajectory.cpp)
through lcbinint_b200.LightCurve and the C ABI, against the reference built
from its sources (oracle/_ref), both reading the same synthetic Earth
ephemeris (tests/ephemeris_fixture.py; the reference's own table is not in its
repository).  The reference loads its ephemeris once per process, so the
comparison runs in a child process with LCBININT_EARTH_EPHEMERIS set.
Bit-identical, except polar inverse-ray points (exact sums here, running sums
in the reference: 1e-12 relative)."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

from ephemeris_fixture import write_ephemeris

ROOT = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.gpu

CHILD = r'''
import ctypes as C, sys
import numpy as np
sys.path.insert(0, ".")
sys.path.insert(0, "tests")
import lcbinint_b200 as lb
from lcbinint_b200 import api
from oracle.oracle import import_reference_module
import test_capi_compat as TC
ref = import_reference_module()

def same(a, b, what):
    a = np.asarray(a); b = np.asarray(b)
    eq = a.view(np.int64) == b.view(np.int64)
    rel = np.abs(a / b - 1.0)
    if not (eq | (rel <= 1e-12)).all() or eq.mean() < 0.9:
        print("MISMATCH", what, int((~eq).sum()), float(np.nanmax(rel)))
        sys.exit(1)

rng = np.random.default_rng(77)
t = np.linspace(9420.0, 9580.0, 120)
modes = [(api.STATIC, ref.STATIC), (api.CIRCULAR, ref.CIRCULAR), (api.KEPLER, ref.KEPLER)]
for coords in ("vbm", "lcbinint"):
    for (mo, mr) in modes:
        p = dict(t0=9500.0 + rng.uniform(-5, 5), tE=float(rng.uniform(20, 40)), u0=float(rng.uniform(-0.15, 0.15)),
                 alpha=float(rng.uniform(0, 6.28)), s=float(rng.uniform(0.7, 1.5)), q=float(np.exp(rng.uniform(-7, 0))),
                 rho=float(np.exp(rng.uniform(np.log(5e-4), np.log(5e-3)))), piEN=float(rng.uniform(-0.5, 0.5)),
                 piEE=float(rng.uniform(-0.5, 0.5)), g1=0.3 / 365.25, g2=-0.4 / 365.25, g3=0.1 / 365.25,
                 lom_szs=0.2, lom_ar=1.5)
        ev = dict(ra=268.5, dec=-29.0, obs_lat=-30.2, obs_lon=-70.8)
        for terrestrial in (False, True):
            ours = lb.LightCurve(options=lb.Options(coordinates=coords), limb_darkening=lb.LimbDarkening.linear(0.4),
                                 orbital_motion_mode=mo, parallax=True, terrestrial_parallax=terrestrial,
                                 event=lb.EventCoordinates(**ev))
            theirs = ref.LightCurve(options=ref.Options(coordinates=coords), limb_darkening=ref.LimbDarkening.linear(0.4),
                                    orbital_motion_mode=mr, parallax=True, terrestrial_parallax=terrestrial,
                                    event=ref.EventCoordinates(**ev))
            same(ours(t, p), theirs(t, p), f"dict {coords} {mo} {terrestrial}")
            same(ours(t, **p), theirs(t, **p), f"keywords {coords} {mo} {terrestrial}")

# xallarap, both parameterisations (dictionary route)
for xtype, extra in (("angular_velocity", dict(xi_1=0.05, xi_2=-0.03, omega_xa=0.02, inc_xa=0.6, phi_xa=1.1)),
                     ("orbital_elements", dict(piEN_xa=0.04, piEE_xa=0.02, period_xa=80.0, ecc_xa=0.2, peri_xa=0.5,
                                               inc_xa=0.7))):
    p = dict(t0=9500.0, tE=25.0, u0=0.08, alpha=0.9, s=1.1, q=3e-3, rho=2e-3, **extra)
    ours = lb.LightCurve(options=lb.Options(xallarap_param_type=xtype), limb_darkening=lb.LimbDarkening.linear(0.3))
    theirs = ref.LightCurve(options=ref.Options(xallarap_param_type=xtype), limb_darkening=ref.LimbDarkening.linear(0.3))
    same(ours(t, p), theirs(t, p), "xallarap " + xtype)

# every result field through the C ABI
O = TC._ours(); R = TC._reference()
P = TC.Params.from_buffer_copy(api.binary_c_params([dict(t0=9500.0, tE=30.0, u0=0.05, alpha=0.4, s=1.05, q=0.02,
                                                         rho=3e-3, piEN=0.2, piEE=0.3)],
                                                   lb.LimbDarkening.linear(0.5), lb.EventCoordinates(ra=270.0, dec=-28.0),
                                                   parallax=True).tobytes())
for vbm in (1, 0):
    o = O.lcbi_default_options(); o.vbm_compatible = vbm
    ra = (TC.Result * len(t))(); rb = (TC.Result * len(t))()
    tt = np.ascontiguousarray(t)
    sa = O.lcbi_magnification_array(tt.ctypes.data, len(t), C.byref(P), C.byref(o), ra)
    sb = R.lcbi_magnification_array(tt.ctypes.data, len(t), C.byref(P), C.byref(o), rb)
    assert sa == sb == 0, (sa, sb)
    for f, _ in TC.Result._fields_:
        x = np.array([getattr(r, f) for r in ra]); y = np.array([getattr(r, f) for r in rb])
        if x.dtype.kind == "f":
            same(x, y, "C ABI " + f)
        else:
            assert np.array_equal(x, y), f
print("OK")
'''


def test_parallax_and_xallarap_match_reference(tmp_path):
    from oracle.oracle import have_reference
    if not have_reference():
        pytest.skip("oracle/_ref not built")
    eph = tmp_path / "earth.txt"
    write_ephemeris(eph)
    env = dict(os.environ, LCBININT_EARTH_EPHEMERIS=str(eph))
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and r.stdout.strip().endswith("OK"), r.stdout[-2000:] + r.stderr[-2000:]


def test_parallax_without_ephemeris_is_a_numerical_error(tmp_path):
    """No table: the first epoch fails (the reference's NaN source)."""
    env = dict(os.environ, LCBININT_EARTH_EPHEMERIS=str(tmp_path / "missing.txt"))
    code = ("import sys, numpy as np; sys.path.insert(0, '.'); import lcbinint_b200 as lb\n"
            "lc = lb.LightCurve(parallax=True)\n"
            "try:\n    lc(np.linspace(0, 1, 5), dict(t0=0.5, tE=1.0, piEN=0.1))\n    print('no error')\n"
            "except RuntimeError as e:\n    print('raised', e)\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert "raised numerical error" in r.stdout, r.stdout + r.stderr
