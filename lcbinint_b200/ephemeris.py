"""A synthetic Earth ephemeris for annual parallax when no JPL Horizons table
is at hand (the reference's own data/earth_orbital_parallax_table.txt is not
in its repository).

`write_synthetic_ephemeris` writes a table in the Horizons vector layout that
both this library and the reference read (JD, x, y, z, vx, vy, vz in AU and
AU/day, equatorial J2000 axes, between $$SOE and $$EOE;
src/lcbinint/model/trajectory.cpp:128-183): the Earth on a Keplerian orbit of
eccentricity 0.0167 in the ecliptic, rotated by the obliquity.  It is smooth
and realistic enough for tests and benchmarks, not a true ephemeris."""
from __future__ import annotations

import math


def write_synthetic_ephemeris(path, jd0: float = 2449500.5, days: float = 12000.0, step: float = 1.0) -> int:
    """Writes states every `step` days from JD `jd0` for `days` days; returns
    how many."""
    ecc, a = 0.0167, 1.000001
    n = 2.0 * math.pi / 365.256363
    obl = math.radians(23.43928)
    peri = math.radians(102.9)
    lines = ["*******************************************************************************",
             "Synthetic Earth ephemeris (Keplerian orbit), Horizons vector-table layout", "$$SOE"]
    count = 0
    t = jd0
    while t <= jd0 + days:
        M = n * (t - 2451547.0)
        E = M
        for _ in range(30):
            E -= (E - ecc * math.sin(E) - M) / (1.0 - ecc * math.cos(E))
        r = a * (1.0 - ecc * math.cos(E))
        nu = 2.0 * math.atan2(math.sqrt(1 + ecc) * math.sin(E / 2), math.sqrt(1 - ecc) * math.cos(E / 2))
        lam = nu + peri
        x, y = r * math.cos(lam), r * math.sin(lam)
        dE = n / (1.0 - ecc * math.cos(E))
        dr = a * ecc * math.sin(E) * dE
        dnu = math.sqrt(1 - ecc * ecc) * dE / (1.0 - ecc * math.cos(E))
        vx = dr * math.cos(lam) - r * math.sin(lam) * dnu
        vy = dr * math.sin(lam) + r * math.cos(lam) * dnu
        X, Y, Z = x, y * math.cos(obl), y * math.sin(obl)
        VX, VY, VZ = vx, vy * math.cos(obl), vy * math.sin(obl)
        lines.append(f"{t:.9f}, A.D. synthetic, {X: .15E}, {Y: .15E}, {Z: .15E}, {VX: .15E}, {VY: .15E}, {VZ: .15E},")
        count += 1
        t += step
    lines += ["$$EOE", "*******************************************************************************"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return count
