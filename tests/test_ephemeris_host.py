"""The Earth-ephemeris loader (host code of the C ABI, no GPU needed): a
Horizons-layout vector table loads with every state between $$SOE and $$EOE,
a missing file raises, and a file without that block loads none.  The table
is process-wide, so the test ends on the empty one, as if none were loaded."""
import pytest


def test_ephemeris_loader(tmp_path):
    from lcbinint_b200.api import set_earth_ephemeris
    from lcbinint_b200.ephemeris import write_synthetic_ephemeris
    path = tmp_path / "earth.txt"
    n = write_synthetic_ephemeris(path, jd0=2459000.5, days=50.0, step=0.5)
    assert n == 101
    assert set_earth_ephemeris(path) == n
    with pytest.raises(FileNotFoundError):
        set_earth_ephemeris(tmp_path / "absent.txt")
    empty = tmp_path / "empty.txt"
    empty.write_text("Horizons header only\nno state block here\n")
    assert set_earth_ephemeris(empty) == 0
