"""The polar lattice's cell-centre angles (lcbinint_b200/csrc/lcbi_trig.cuh).

The reference evaluates cos and sin of each polar cell's angle with the host
C library (finite_source_magnifier.cpp:1198-1203); the device uses its own
correctly rounded sin and cos, compiled here for the host from the same
header.  Checked against 300-bit values (mpmath) on the polar lattices'
angles (phi = (i + 1/2) 2 pi / P) and on random angles, including those where
the host library itself rounds the other way (the exact value within about
0.014 units in the last place of a rounding midpoint, about 0.13% of
arguments with this C library).  The constants are checked against the
generator that made them."""
import ctypes
import math
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "lcbinint_b200" / "csrc"


@pytest.fixture(scope="module")
def trig(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    so = tmp_path_factory.mktemp("trig") / "libtrig.so"
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", f"-I{CSRC}",
           str(ROOT / "tests" / "cpp" / "trig_driver.cpp"), "-o", str(so)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lib = ctypes.CDLL(str(so))
    lib.trig_sincos_cr.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 3

    def f(x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        s = np.empty_like(x)
        c = np.empty_like(x)
        lib.trig_sincos_cr(x.size, x.ctypes.data, s.ctypes.data, c.ctypes.data)
        return s, c
    return f


def _angles(n, seed=5):
    rng = np.random.default_rng(seed)
    P = rng.integers(16, 5_000_000, n)
    i = rng.integers(0, P)
    lattice = (i.astype(np.float64) + 0.5) * (2.0 * math.pi / P.astype(np.float64))
    quarter = np.array([(m + 0.5) * (2.0 * math.pi / P) for P in (18, 4_363_718, 4_363_722) for m in
                        (P // 4 - 1, P // 4, P // 2, 3 * P // 4)])
    return np.concatenate([lattice, rng.uniform(0.0, 2.0 * math.pi, n), quarter, [0.0, 1e-300, 1e-8]])


def test_correctly_rounded(trig):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 300
    x = _angles(4000)
    s, c = trig(x)
    for xi, si, ci in zip(x, s, c):
        X = mpmath.mpf(float(xi))
        assert si == float(mpmath.sin(X)), float.hex(float(xi))
        assert ci == float(mpmath.cos(X)), float.hex(float(xi))


def test_agrees_with_host_library_except_its_misroundings(trig):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 300
    x = _angles(100_000, seed=9)
    s, c = trig(x)
    gs = np.array([math.sin(v) for v in x])
    gc = np.array([math.cos(v) for v in x])
    differ = np.nonzero((s != gs) | (c != gc))[0]
    assert differ.size <= 0.005 * x.size
    for k in differ:
        X = mpmath.mpf(float(x[k]))
        assert s[k] == float(mpmath.sin(X)) and c[k] == float(mpmath.cos(X))


def test_constants_match_generator():
    pytest.importorskip("mpmath")
    out = subprocess.run(["python", str(CSRC / "gen_trig_constants.py")], capture_output=True, text=True,
                         check=True).stdout
    header = (CSRC / "lcbi_trig.cuh").read_text()
    for line in out.splitlines():
        line = line.strip()
        if line.startswith("constexpr"):
            assert line in header, line
        elif line.startswith("{"):
            hi, lo = line.strip("{},").split(", ")
            assert hi in header, line
            if float.fromhex(lo) != 0.0 and abs(float.fromhex(hi)) > 2.0 ** -45:
                assert lo in header, line
