"""LightCurve.source_trajectory (python/lcbinint_pybind.cpp:3292-3330) against
the reference's own module built from its sources (oracle/_ref).

Host arithmetic only (no GPU): the straight-line trajectory in both coordinate
conventions, lens orbital motion (circular and Keplerian) turning it into the
binary's frame, and annual plus terrestrial parallax on the synthetic Earth
ephemeris (tests/ephemeris_fixture.py) that both sides read.  The reference
loads its ephemeris once per process, so the comparison runs in a child
process with LCBININT_EARTH_EPHEMERIS set.  Bar: bit-identical positions."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

from ephemeris_fixture import write_ephemeris

ROOT = Path(__file__).resolve().parents[1]

CHILD = r'''
import sys
import numpy as np
sys.path.insert(0, ".")
import lcbinint_b200 as lb
from lcbinint_b200 import api
from oracle.oracle import import_reference_module
ref = import_reference_module()

def same(a, b, what):
    a = np.asarray(a, dtype=np.float64); b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape or not np.array_equal(a.view(np.int64), b.view(np.int64)):
        print("MISMATCH", what, a[:3], b[:3])
        sys.exit(1)

rng = np.random.default_rng(5)
t = np.linspace(9420.0, 9580.0, 57)
modes = [(api.STATIC, ref.STATIC), (api.CIRCULAR, ref.CIRCULAR), (api.KEPLER, ref.KEPLER)]
n = 0
for coords in ("vbm", "lcbinint"):
    for (mo, mr) in modes:
        for parallax in (False, True):
            p = dict(t0=9500.0 + rng.uniform(-5, 5), tE=float(rng.uniform(20, 40)),
                     u0=float(rng.uniform(-0.15, 0.15)), alpha=float(rng.uniform(0, 6.28)),
                     s=float(rng.uniform(0.7, 1.5)), q=float(np.exp(rng.uniform(-7, 0))),
                     g1=0.3 / 365.25, g2=-0.4 / 365.25, g3=0.1 / 365.25, lom_szs=0.2, lom_ar=1.5)
            if parallax:
                p.update(piEN=float(rng.uniform(-0.5, 0.5)), piEE=float(rng.uniform(-0.5, 0.5)))
            ev = dict(ra=268.5, dec=-29.0, obs_lat=-30.2, obs_lon=-70.8, tfix=9500.0)
            ours = lb.LightCurve(options=lb.Options(coordinates=coords), orbital_motion_mode=mo, parallax=parallax,
                                 event=lb.EventCoordinates(**ev))
            theirs = ref.LightCurve(options=ref.Options(coordinates=coords), orbital_motion_mode=mr,
                                    parallax=parallax, event=ref.EventCoordinates(**ev))
            for route, a, b in (("dict", ours.source_trajectory(t, p), theirs.source_trajectory(t, p)),
                                ("keywords", ours.source_trajectory(t, **p), theirs.source_trajectory(t, **p))):
                what = f"{route} {coords} mode={mo} parallax={parallax}"
                same(a.times, b.times, what + " times")
                same(a.x, b.x, what + " x")
                same(a.y, b.y, what + " y")
                n += 1
# A dictionary's parallax components count even without parallax=True.
q = dict(t0=9500.0, tE=30.0, u0=0.1, alpha=0.3, s=1.1, q=0.01, piEN=0.2, piEE=-0.1)
a = lb.LightCurve().source_trajectory(t, q)
b = ref.LightCurve().source_trajectory(t, q)
same(a.x, b.x, "dict parallax without flag")
# As keywords they need the flag, on both sides.
for mod in (lb, ref):
    try:
        mod.LightCurve().source_trajectory(t, t0=0.0, piEN=0.1)
    except (ValueError, RuntimeError):
        pass
    else:
        print("MISMATCH keywords without parallax accepted by", mod.__name__)
        sys.exit(1)
assert lb.LightCurve().source_trajectory([], dict(t0=0.0)).x == []
print("OK", n)
'''


def test_source_trajectory_matches_reference(tmp_path):
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import import_reference_module
    if import_reference_module() is None:
        pytest.skip("the reference module is not built (make -C oracle ref)")
    eph = tmp_path / "earth.txt"
    write_ephemeris(str(eph))
    env = dict(os.environ, LCBININT_EARTH_EPHEMERIS=str(eph))
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
