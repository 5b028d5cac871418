"""Generates the golden fixtures in tests/golden/ from the reference itself.

    make -C oracle && python tests/golden/make_golden.py

The values come from the reference lcbinint compiled from its own sources
(oracle/_ref, see oracle/Makefile) on seeded synthetic inputs.  The reference
tree is only needed here, when (re)generating; the committed .npz files are
what the tests read, on any machine.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import Reference, default_settings  # noqa: E402

OUT = Path(__file__).resolve().parent


def point_source(ref: Reference):
    """2,000 point-source magnifications, the 1e6-point batch's distribution (seed 10)."""
    rng = np.random.default_rng(10)
    n = 2000
    y = rng.uniform(-1.5, 1.5, (n, 2))
    s = np.exp(rng.uniform(np.log(0.3), np.log(3.0), n))
    q = np.exp(rng.uniform(np.log(1e-5), 0.0, n))
    A, nimg = ref.binary_mag0(s, q, y[:, 0], y[:, 1])
    Ad, nd, ind = ref.binary_mag0_derivatives(s, q, y[:, 0], y[:, 1])
    np.savez_compressed(OUT / "point_source.npz", s=s, q=q, y1=y[:, 0], y2=y[:, 1], A=A, nimg=nimg,
                        indicator=ind)


def finite_source(ref: Reference):
    """Forced inverse-ray magnifications (lcbinint.binary_inverse_ray semantics) on
    near-caustic sources, Cartesian and polar, uniform and limb-darkened (seed 11)."""
    rng = np.random.default_rng(11)
    rows = []
    cases = [
        # s, q_core, rho, ld_c
        (0.95, 100.0, 5e-3, 0.5),
        (1.0, 10.0, 1e-2, 0.0),
        (0.7, 1.0 / 0.3, 2e-2, 0.3),
        (1.5, 1.0, 1e-2, 0.0),
    ]
    for s, q, rho, c in cases:
        br, bbox, _ = ref.caustic_cache(s, q, 1400)
        pts = br.reshape(-1, 2)
        for k in range(6):
            p = pts[rng.integers(len(pts))]
            x, y = p + rng.normal(0.0, rho, 2)
            for mode, nbin in ((1, 20), (2, 20)):
                st = default_settings(source_bins=nbin, finite_mode=mode, limb_darkening_c=c)
                A, m = ref.inverse_ray(st, s, q, x, y, rho)
                rows.append((s, q, x, y, rho, c, mode, nbin, A[0], m[0]))
    a = np.array(rows)
    np.savez_compressed(OUT / "inverse_ray.npz", s=a[:, 0], q=a[:, 1], x=a[:, 2], y=a[:, 3], rho=a[:, 4],
                        ld_c=a[:, 5], mode=a[:, 6].astype(np.int32), nbin=a[:, 7].astype(np.int32),
                        A=a[:, 8], method=a[:, 9].astype(np.int32))


def light_curve(ref: Reference):
    """The README light curve (200 epochs, nbin 50, linear LD 0.5, VBM coordinates),
    auto grid and Cartesian-forced."""
    times = np.linspace(-0.5, 0.5, 200)
    p = dict(t0=0.0, tE=1.0, u0=-0.01, alpha=0.5, s=0.95, q=1e-2, rho=5e-3)
    out = {}
    for name, mode in (("auto", 4), ("cartesian", 1)):
        st = default_settings(source_bins=50, finite_mode=mode, limb_darkening_c=0.5)
        A, m, rc = ref.light_curve_static(st, times, **p)
        assert rc == 0
        out[f"A_{name}"] = A
        out[f"method_{name}"] = m
    np.savez_compressed(OUT / "light_curve_readme.npz", times=times, **out)


if __name__ == "__main__":
    ref = Reference()
    point_source(ref)
    finite_source(ref)
    light_curve(ref)
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)
