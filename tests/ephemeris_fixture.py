"""A synthetic Earth ephemeris in the JPL Horizons vector-table layout the
reference reads (src/lcbinint/model/trajectory.cpp:128-183), for parallax
tests: the reference's own table is not in its repository.  The Earth moves
on a slightly eccentric Keplerian orbit in the ecliptic, rotated into
equatorial coordinates; the numbers only need to be smooth and realistic, not
true ephemerides."""
import math


def write_ephemeris(path, jd0=2458000.5, days=4000, step=1.0):
    ecc, a = 0.0167, 1.000001
    n = 2.0 * math.pi / 365.256363
    obl = math.radians(23.43928)
    peri = math.radians(102.9)
    lines = ["*******************************************************************************",
             "Synthetic ephemeris for tests", "$$SOE"]
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
        t += step
    lines += ["$$EOE", "*******************************************************************************"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
