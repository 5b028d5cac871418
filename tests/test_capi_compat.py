"""The reference's own C ABI (include/lcbinint/lcbinint.h) served by the GPU library.

* CPU: the structs declared in include/lcbinint_b200.h have the reference's
  layout (compiled side by side with the reference header, when present), and
  the defaults match.
* GPU: the known answers of the reference's unit test
  (tests/unit/test_core.cpp:56-106), and bit-for-bit agreement of every result
  field with the compiled reference (oracle/_ref) on random static binaries in
  both coordinate conventions, point and finite source.
"""
import ctypes as C
import math
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
REF_INCLUDE = Path(os.environ.get("LCBININT_REFERENCE", "/root/reference")) / "include"


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "t0", "tE", "umin", "q", "sep", "theta", "rho", "omega", "piEN", "piEE", "piEN_xa", "piEE_xa", "ra_xa",
        "dec_xa", "period_xa", "ecc_xa", "peri_xa", "v_sep", "q2", "sep2", "ang", "ra", "dec", "earth_axis", "tfix",
        "obs_lat", "obs_lon", "limb_darkening_c", "limb_darkening_d")] + [("orbital_motion_mode", C.c_int)] + \
        [(n, C.c_double) for n in ("g1", "g2", "g3", "lom_szs", "lom_ar", "xi_1", "xi_2", "omega_xa", "inc_xa",
                                   "phi_xa")]


class Options(C.Structure):
    _fields_ = [("parallax_mode", C.c_int), ("orbit_pair", C.c_int), ("center_of_mass", C.c_int),
                ("caustic_bins", C.c_int), ("source_bins", C.c_int), ("mode", C.c_int), ("vbm_compatible", C.c_int),
                ("xallarap_param_type", C.c_int), ("grid_ratio", C.c_double), ("polar_source_bins", C.c_int),
                ("polar_grid_ratio", C.c_double), ("point_source_threshold", C.c_double),
                ("hexadecapole_threshold", C.c_double), ("adaptive_hex_threshold", C.c_double),
                ("adaptive_source_bins", C.c_int), ("max_source_bins", C.c_int), ("finite_source_tol", C.c_double),
                ("finite_source_reltol", C.c_double)]


class Result(C.Structure):
    _fields_ = [("magnification", C.c_double), ("point_source_magnification", C.c_double),
                ("finite_source_magnification", C.c_double), ("source_x", C.c_double), ("source_y", C.c_double),
                ("image_count", C.c_int), ("finite_source_error_estimate", C.c_double),
                ("finite_source_refinement_level", C.c_int), ("finite_source_converged", C.c_int)]


def _declare(L):
    L.lcbi_default_params.restype = Params
    L.lcbi_default_options.restype = Options
    L.lcbi_magnification.argtypes = [C.c_double, C.POINTER(Params), C.POINTER(Options), C.POINTER(Result)]
    L.lcbi_magnification.restype = C.c_int
    L.lcbi_magnification_array.argtypes = [C.c_void_p, C.c_int, C.POINTER(Params), C.POINTER(Options), C.c_void_p]
    L.lcbi_magnification_array.restype = C.c_int
    L.lcbi_status_string.argtypes = [C.c_int]
    L.lcbi_status_string.restype = C.c_char_p
    return L


def _ours():
    from lcbinint_b200 import _lib
    return _declare(_lib.lib())


def _reference():
    from oracle.oracle import REF_SO, have_reference
    if not have_reference():
        pytest.skip("oracle/_ref not built")
    return _declare(C.CDLL(str(REF_SO)))


_LAYOUT_C = r"""
#include <stdio.h>
#include <stddef.h>
#include HEADER
#define F(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  printf("params %zu options %zu result %zu\n", sizeof(lcbi_params), sizeof(lcbi_options), sizeof(lcbi_result));
  F(lcbi_params, orbital_motion_mode) F(lcbi_params, g1) F(lcbi_params, phi_xa) F(lcbi_params, limb_darkening_d)
  F(lcbi_options, xallarap_param_type) F(lcbi_options, grid_ratio) F(lcbi_options, finite_source_reltol)
  F(lcbi_options, adaptive_source_bins) F(lcbi_result, image_count) F(lcbi_result, finite_source_error_estimate)
  F(lcbi_result, finite_source_converged)
  return 0;
}
"""


def _layout(tmp_path, header):
    src = tmp_path / "layout.c"
    src.write_text(_LAYOUT_C.replace("HEADER", f'"{header}"'))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    return subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout


def test_struct_layout_matches_reference_header(tmp_path):
    ref_h = REF_INCLUDE / "lcbinint" / "lcbinint.h"
    if not ref_h.exists() or shutil.which("gcc") is None:
        pytest.skip("reference header or gcc not available")
    ours = _layout(tmp_path, ROOT / "include" / "lcbinint_b200.h")
    ref = _layout(tmp_path, ref_h)
    assert ours == ref
    # ...and the ctypes mirrors used by the GPU tests agree with it.
    sizes = ours.splitlines()[0].split()
    assert int(sizes[1]) == C.sizeof(Params) and int(sizes[3]) == C.sizeof(Options)
    assert int(sizes[5]) == C.sizeof(Result)


def test_record_dtypes_match_the_structs():
    """The numpy records lcbinint_b200 passes to lcbi_gpu_magnification_arrays
    have the structs' sizes and field offsets."""
    from lcbinint_b200 import _lib
    for dt, st in ((_lib.PARAMS_DTYPE, Params), (_lib.OPTIONS_DTYPE, Options), (_lib.RESULT_DTYPE, Result)):
        assert dt.itemsize == C.sizeof(st)
        for name, _ in st._fields_:
            assert dt.fields[name][1] == getattr(st, name).offset, name
    d = _lib.default_params(1)[0]
    assert (d["tE"], d["q"], d["sep"], d["lom_ar"], d["orbital_motion_mode"]) == (1.0, 1.0, 1.0, 1.0, 0)
    o = _lib.default_options()[0]
    assert (o["caustic_bins"], o["source_bins"], o["mode"], o["orbit_pair"], o["max_source_bins"]) == \
        (1400, 50, 4, 23, 400)


def test_defaults_and_status_strings():
    L = _ours()
    p = L.lcbi_default_params()
    o = L.lcbi_default_options()
    assert p.tE == 1.0 and p.q == 1.0 and p.sep == 1.0 and p.lom_ar == 1.0 and p.orbital_motion_mode == 0
    assert (o.caustic_bins, o.source_bins, o.mode, o.orbit_pair, o.max_source_bins) == (1400, 50, 4, 23, 400)
    assert (o.grid_ratio, o.point_source_threshold, o.hexadecapole_threshold, o.adaptive_hex_threshold) == \
        (4.0, 20.0, 3.0, 0.001)
    assert [L.lcbi_status_string(i) for i in range(4)] == [b"ok", b"invalid argument", b"numerical error",
                                                            b"unsupported"]


@pytest.mark.gpu
def test_reference_unit_test_known_answers():
    """tests/unit/test_core.cpp:56-106 of the reference."""
    L = _ours()
    p = L.lcbi_default_params()
    o = L.lcbi_default_options()
    r = Result()
    assert L.lcbi_magnification(0.0, C.byref(p), C.byref(o), C.byref(r)) == 0
    assert abs(r.source_x) <= 1e-12 and abs(r.source_y) <= 1e-12
    p.umin, p.theta, p.q, p.sep = 0.1, 0.0, 0.1, 1.0
    assert L.lcbi_magnification(0.2, C.byref(p), C.byref(o), C.byref(r)) == 0
    assert abs(r.source_x - 0.2) <= 1e-12 and abs(r.source_y - 0.1) <= 1e-12
    assert abs(r.magnification - 5.871444912771214) <= 1e-10
    p.sep, p.q = 1.5, 1.0
    assert L.lcbi_magnification(0.2, C.byref(p), C.byref(o), C.byref(r)) == 0
    assert abs(r.magnification - 3.5659775904852786) <= 1e-10
    p.sep, p.q, p.umin, p.rho = 1.0, 0.1, 1.1, 0.001
    o.center_of_mass = 1
    assert L.lcbi_magnification(1.2, C.byref(p), C.byref(o), C.byref(r)) == 0
    assert math.isfinite(r.finite_source_magnification)


@pytest.mark.gpu
def test_invalid_and_unsupported_input():
    L = _ours()
    o = L.lcbi_default_options()
    r = Result()
    p = L.lcbi_default_params()
    p.tE = 0.0
    assert L.lcbi_magnification(0.0, C.byref(p), C.byref(o), C.byref(r)) == 1
    p = L.lcbi_default_params()
    p.piEN = 0.1  # annual parallax without an Earth ephemeris: a NaN source, as in the reference
    if not os.environ.get("LCBININT_EARTH_EPHEMERIS"):
        assert L.lcbi_magnification(0.0, C.byref(p), C.byref(o), C.byref(r)) == 2
    p = L.lcbi_default_params()
    p.q2 = 0.1  # triple lenses are not built
    assert L.lcbi_magnification(0.0, C.byref(p), C.byref(o), C.byref(r)) == 3
    p = L.lcbi_default_params()
    p.omega = 0.1  # unsupported in the reference too
    assert L.lcbi_magnification(0.0, C.byref(p), C.byref(o), C.byref(r)) == 3
    assert math.isnan(r.magnification)
    assert L.lcbi_magnification_array(None, 0, C.byref(p), C.byref(o), None) == 0
    assert L.lcbi_magnification_array(None, -1, C.byref(p), C.byref(o), None) == 1


def _fields(results):
    return {f: np.array([getattr(r, f) for r in results]) for f, _ in Result._fields_}


@pytest.mark.gpu
@pytest.mark.parametrize("vbm,com,rho,mode", [(1, 0, 0.0, 4), (0, 0, 0.0, 4), (1, 0, 4e-3, 4), (0, 0, 6e-3, 1),
                                              (0, 1, 3e-3, 2), (1, 0, 1e-2, 4)])
def test_matches_compiled_reference_bit_for_bit(vbm, com, rho, mode):
    ours = _ours()
    ref = _reference()
    rng = np.random.default_rng(100 + 10 * vbm + com + int(rho * 1e4) + mode)
    for _ in range(3):
        p = ours.lcbi_default_params()
        o = ours.lcbi_default_options()
        p.t0 = float(rng.uniform(-0.1, 0.1))
        p.tE = float(rng.uniform(0.5, 2.0))
        p.umin = float(rng.uniform(-0.15, 0.15))
        p.theta = float(rng.uniform(0.0, 2.0 * np.pi))
        p.sep = float(np.exp(rng.uniform(np.log(0.5), np.log(2.0))))
        p.q = float(np.exp(rng.uniform(np.log(1e-3), np.log(1.0))))
        if vbm and rng.random() < 0.5:
            p.q = 1.0 / p.q
        p.rho = rho
        p.limb_darkening_c = float(rng.uniform(0.0, 0.7))
        o.vbm_compatible = vbm
        o.center_of_mass = com
        o.mode = mode
        o.source_bins = 30
        times = np.ascontiguousarray(np.linspace(p.t0 - 1.5 * p.tE, p.t0 + 1.5 * p.tE, 60))
        a = (Result * len(times))()
        b = (Result * len(times))()
        ra = ours.lcbi_magnification_array(times.ctypes.data, len(times), C.byref(p), C.byref(o), a)
        rb = ref.lcbi_magnification_array(times.ctypes.data, len(times), C.byref(p), C.byref(o), b)
        assert ra == rb
        fa, fb = _fields(a), _fields(b)
        for f in fa:
            x, y = fa[f], fb[f]
            if x.dtype.kind == "f":
                assert np.array_equal(np.isnan(x), np.isnan(y)), f
                ok = ~np.isnan(x)
                assert np.array_equal(x[ok].view(np.int64), y[ok].view(np.int64)), \
                    (f, np.nanmax(np.abs(x / y - 1.0)))
            else:
                assert np.array_equal(x, y), f


@pytest.mark.gpu
@pytest.mark.parametrize("mode,vbm,rho", [(1, 1, 0.0), (1, 0, 3e-3), (2, 1, 5e-3), (2, 0, 0.0)])
def test_orbital_motion_matches_compiled_reference(mode, vbm, rho):
    """Circular (1) and Keplerian (2) lens orbital motion through the C ABI,
    over 200 days, bit for bit against the compiled reference."""
    ours = _ours()
    ref = _reference()
    rng = np.random.default_rng(200 + 10 * mode + vbm)
    for _ in range(2):
        p = ours.lcbi_default_params()
        o = ours.lcbi_default_options()
        p.t0 = 0.0
        p.tE = float(rng.uniform(15.0, 40.0))
        p.umin = float(rng.uniform(-0.2, 0.2))
        p.theta = float(rng.uniform(0.0, 2.0 * np.pi))
        p.sep = float(np.exp(rng.uniform(np.log(0.6), np.log(1.6))))
        p.q = float(np.exp(rng.uniform(np.log(1e-3), 0.0)))
        p.rho = rho
        p.limb_darkening_c = 0.4
        p.orbital_motion_mode = mode
        p.g1 = float(rng.uniform(-1.0, 1.0)) / 365.25
        p.g2 = float(rng.uniform(-1.0, 1.0)) / 365.25
        p.g3 = float(rng.uniform(0.0, 0.5)) / 365.25
        if mode == 2:
            p.lom_szs = float(rng.uniform(-0.5, 0.5))
            p.lom_ar = float(rng.uniform(1.0, 2.0))
        o.vbm_compatible = vbm
        o.source_bins = 30
        times = np.ascontiguousarray(np.linspace(-100.0, 100.0, 80))
        a = (Result * len(times))()
        b = (Result * len(times))()
        ra = ours.lcbi_magnification_array(times.ctypes.data, len(times), C.byref(p), C.byref(o), a)
        rb = ref.lcbi_magnification_array(times.ctypes.data, len(times), C.byref(p), C.byref(o), b)
        assert ra == rb
        fa, fb = _fields(a), _fields(b)
        for f in fa:
            x, y = fa[f], fb[f]
            if x.dtype.kind == "f":
                assert np.array_equal(np.isnan(x), np.isnan(y)), f
                ok = ~np.isnan(x)
                assert np.array_equal(x[ok].view(np.int64), y[ok].view(np.int64)), \
                    (f, np.nanmax(np.abs(x / y - 1.0)))
            else:
                assert np.array_equal(x, y), f
