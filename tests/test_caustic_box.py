"""The outer caustic box (caustic_outer_box in csrc/lcbi_caustic.cuh) holds
the reference's sampled caustic.

Points whose source lies outside that box by the decision's margin take the
bounding-box exit of the finite-source decision
(src/lcbinint/magnification/finite_source_magnifier.cpp:4679-4698) without
their caustic being sampled, which is only right if the box contains the
bounding box of the reference's 1,400-phase caustic samples.  The box is
restated here in numpy, step for step, and checked against the samples of the
reference compiled from source (oracle/_ref) over separations 0.1-10 and mass
ratios 1e-6-1 in both conventions.  CPU only.
"""
import numpy as np
import pytest


def _disc(mn, mf, s, zn, shift):
    dmax = np.sqrt(2.0 * mn)
    dfmin = max(s - dmax, s / (1.0 + np.sqrt(mn / mf)))
    e = mf / (dfmin * dfmin)
    dmin = np.sqrt(mn / (1.0 + e))
    if e < 1.0:
        dmax = min(dmax, np.sqrt(mn / (1.0 - e)))
    core = max(abs(dmin - mn / dmin), abs(dmax - mn / dmax))
    c, r = zn, core + mf / dfmin
    if dmax < s:
        r2 = core + mf * dmax / (s * (s - dmax))
        if r2 < r:
            c, r = zn - shift, r2
    return c, r


def outer_box(separation, mass_ratio):
    s, q_in = abs(separation), abs(mass_ratio)
    q = q_in if q_in < 1.0 else 1.0 / q_in
    a = -s if q_in < 1.0 else s
    m1 = 1.0 / (1.0 + q)
    m2 = q * m1
    c1, r1 = _disc(m1, m2, s, a, m2 / a)
    c2, r2 = _disc(m2, m1, s, 0.0, -m1 / a)
    r1 = r1 * (1.0 + 1.0e-6) + 1.0e-9
    r2 = r2 * (1.0 + 1.0e-6) + 1.0e-9
    sh = a * m1
    lo, hi = min(c1 - r1, c2 - r2) - sh, max(c1 + r1, c2 + r2) - sh
    pad = 1.0e-9 + 1.0e-9 * (abs(lo) + abs(hi))
    return lo - pad, hi + pad, max(r1, r2)


def test_outer_box_contains_the_reference_caustic_samples():
    from oracle.oracle import Reference, have_reference
    if not have_reference():
        pytest.skip("oracle/_ref not built")
    ref = Reference()
    rng = np.random.default_rng(21)
    cases = [(1.0, 1.0), (1.0, 1e-6), (0.1, 1e-6), (10.0, 1e-6), (0.1, 1.0), (10.0, 1.0), (0.7, 0.3), (1.4, 2e-4)]
    cases += [(float(np.exp(rng.uniform(np.log(0.1), np.log(10.0)))), float(np.exp(rng.uniform(np.log(1e-6), 0.0))))
              for _ in range(150)]
    widths = []
    for s, q in cases:
        for q_arg in (q, 1.0 / q):
            branches, bbox, _ = ref.caustic_cache(s, q_arg, 1400)
            pts = branches.reshape(-1, 2)
            pts = pts[np.isfinite(pts).all(axis=1)]
            lo, hi, half_y = outer_box(s, q_arg)
            assert pts[:, 0].min() >= lo and pts[:, 0].max() <= hi, (s, q_arg)
            assert np.abs(pts[:, 1]).max() <= half_y, (s, q_arg)
            widths.append((hi - lo) / max(pts[:, 0].max() - pts[:, 0].min(), 1e-12))
    # It is a bound, not the box itself, but not a vacuous one either.
    assert np.median(widths) < 20.0
