"""CPU tests: the oracle restatement against the reference's golden vectors.

These pin the oracle before it is trusted as the checker of the GPU path:
  * the reference's own known-answer values (tests/regression/test_vbm_consistency.py:8-13,
    VBMicrolensing BinaryMag0 values lcbinint matches to 1e-10);
  * fixtures generated from the reference compiled from source (tests/golden/make_golden.py),
    which the oracle must reproduce bit for bit;
  * the root-solver known-answer checks of tests/unit/test_core.cpp:112-155.
"""
import math

import numpy as np
import pytest

# (s, q, y1, y2, A) -- tests/regression/test_vbm_consistency.py:8-13
BINARY_POINT_CASES = [
    (1.0, 0.1, 0.2, 0.1, 5.871444912771214),
    (0.7, 0.3, -0.4, 0.2, 2.116643550532278),
    (1.5, 1.0, 0.05, -0.2, 1.5493462433112466),
    (1.0, 1.0e-3, 0.3, 0.4, 2.1789388609029046),
]


@pytest.mark.parametrize("s,q,y1,y2,expected", BINARY_POINT_CASES)
def test_oracle_point_source_known_answers(oracle_lib, s, q, y1, y2, expected):
    A, nimg = oracle_lib.binary_mag0([s], [q], [y1], [y2])
    assert math.isclose(A[0], expected, rel_tol=1e-10, abs_tol=1e-11)
    assert nimg[0] in (3, 5)


def test_oracle_point_source_bit_exact_vs_reference_fixture(oracle_lib, golden):
    g = golden("point_source.npz")
    A, nimg = oracle_lib.binary_mag0(g["s"], g["q"], g["y1"], g["y2"])
    assert np.array_equal(A.view(np.int64), g["A"].view(np.int64))
    assert np.array_equal(nimg, g["nimg"])
    Ad, nd, ind = oracle_lib.binary_mag0_derivatives(g["s"], g["q"], g["y1"], g["y2"])
    assert np.array_equal(ind.view(np.int64), g["indicator"].view(np.int64))


def _poly_eval(coef, z):
    v = 0j
    for c in coef[::-1]:
        v = v * z + c
    return v


@pytest.mark.parametrize("coef", [
    [-1.0, 0.0, 0.0, 1.0],
    [complex(-1.0, 0.25), complex(0.5, -0.75), -1.0, complex(0.25, 0.5), -0.25, 1.0],
])
def test_oracle_roots_known_answers(oracle_lib, coef):
    # tests/unit/test_core.cpp:112-155: every root satisfies |p(z)| < 1e-9.
    roots = oracle_lib.roots(coef)
    assert roots.size == len(coef) - 1
    for z in roots:
        assert abs(_poly_eval(np.asarray(coef, dtype=complex), z)) < 1e-9


def test_oracle_matches_live_reference_roots(oracle_lib, ref_lib):
    rng = np.random.default_rng(3)
    for deg in (3, 4, 5):
        for _ in range(200):
            c = rng.normal(size=deg + 1) + 1j * rng.normal(size=deg + 1)
            a = oracle_lib.roots(c)
            b = ref_lib.roots(c)
            assert np.array_equal(a.view(np.float64), b.view(np.float64))
