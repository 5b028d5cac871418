"""The synthetic Earth ephemeris of lcbinint_b200.ephemeris, for the parallax
tests (the reference's own table is not in its repository)."""
from lcbinint_b200.ephemeris import write_synthetic_ephemeris


def write_ephemeris(path):
    return write_synthetic_ephemeris(path)
