"""ctypes access to the CPU oracle libraries (test infrastructure only).

Two libraries live under ``oracle/``:

* ``_build/liblcbi_oracle.so`` -- this repository's CPU restatement of the
  reference algorithm (``oracle_ps.cpp``, ``oracle_fs.cpp``);
* ``_ref/liblcbi_ref.so`` -- the reference lcbinint compiled from its own
  sources plus a C shim (``ref_shim.cpp``, built by ``oracle/Makefile``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU arms of ``bench.py``
import this module.  The product (``lcbinint_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liblcbi_oracle.so"
REF_SO = HERE / "_ref" / "liblcbi_ref.so"
REF_DIR = HERE / "_ref"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class FsSettings(C.Structure):
    """Flat mirror of FiniteSourceSettings (finite_source_magnifier.hpp:22-38)."""

    _fields_ = [
        ("source_bins", C.c_int),
        ("caustic_bins", C.c_int),
        ("grid_ratio", C.c_double),
        ("polar_source_bins", C.c_int),
        ("polar_grid_ratio", C.c_double),
        ("finite_mode", C.c_int),
        ("kinji_threshold", C.c_double),
        ("hex_threshold", C.c_double),
        ("adaptive_hex_threshold", C.c_double),
        ("limb_darkening_c", C.c_double),
        ("limb_darkening_d", C.c_double),
        ("adaptive_source_bins", C.c_int),
        ("max_source_bins", C.c_int),
        ("finite_source_tol", C.c_double),
        ("finite_source_reltol", C.c_double),
    ]


def default_settings(**kw) -> FsSettings:
    s = FsSettings(
        source_bins=50, caustic_bins=1400, grid_ratio=4.0, polar_source_bins=0,
        polar_grid_ratio=0.0, finite_mode=1, kinji_threshold=20.0, hex_threshold=3.0,
        adaptive_hex_threshold=0.001, limb_darkening_c=0.0, limb_darkening_d=0.0,
        adaptive_source_bins=0, max_source_bins=400, finite_source_tol=0.0,
        finite_source_reltol=0.0)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


class _Lib:
    def __init__(self, path: Path, prefix: str):
        if not path.exists():
            raise FileNotFoundError(f"oracle library missing: {path} (run `make -C oracle`)")
        self.lib = C.CDLL(str(path))
        self.p = prefix

    def fn(self, name):
        return getattr(self.lib, self.p + name)

    def binary_mag0(self, s, q, x, y):
        s, q, x, y = (_f64(np.broadcast_to(v, np.broadcast(s, q, x, y).shape)).ravel()
                      for v in (s, q, x, y))
        n = s.size
        A = np.empty(n)
        nimg = np.empty(n, dtype=np.int32)
        self.fn("binary_mag0_many")(n, _ptr(s), _ptr(q), _ptr(x), _ptr(y), _ptr(A), _ptr(nimg, _ip))
        return A, nimg

    def binary_mag0_derivatives(self, s, q, x, y):
        s, q, x, y = (_f64(np.broadcast_to(v, np.broadcast(s, q, x, y).shape)).ravel()
                      for v in (s, q, x, y))
        n = s.size
        A = np.empty(n)
        ind = np.empty(n)
        nimg = np.empty(n, dtype=np.int32)
        self.fn("binary_mag0_derivatives_many")(n, _ptr(s), _ptr(q), _ptr(x), _ptr(y), _ptr(A),
                                                _ptr(nimg, _ip), _ptr(ind))
        return A, nimg, ind

    def image_candidates(self, s, q, x, y):
        out = np.zeros(25)
        n = self.fn("image_candidates")(C.c_double(s), C.c_double(q), C.c_double(x),
                                        C.c_double(y), _ptr(out))
        return out[: 5 * n].reshape(n, 5)

    def roots(self, coef, polish=True):
        coef = np.asarray(coef, dtype=np.complex128)
        deg = coef.size - 1
        c = _f64(np.stack([coef.real, coef.imag], axis=1).ravel())
        r = np.zeros(2 * deg)
        self.fn("roots")(_ptr(c), deg, _ptr(r), int(polish))
        return r[0::2] + 1j * r[1::2]


class _FsLib(_Lib):
    """Finite-source entry points shared by the oracle and the reference shim."""

    def __init__(self, path, prefix):
        super().__init__(path, prefix)
        f = self.fn
        st = C.POINTER(FsSettings)
        f("binary_mag").argtypes = [st] + [C.c_double] * 6 + [C.c_int, _dp, _ip]
        f("inverse_ray_many").argtypes = [st, C.c_int] + [_dp] * 6 + [_ip]
        if prefix == "orc_":
            f("inverse_ray_many_fixed").argtypes = [st, C.c_int] + [_dp] * 6 + [_ip, _dp, C.c_void_p]
        f("seeds").argtypes = [st] + [C.c_double] * 5 + [_dp, C.c_int]
        f("cartesian").argtypes = [st] + [C.c_double] * 5 + [_dp, C.c_int, _dp]
        f("cartesian").restype = C.c_double
        f("polar").argtypes = [st] + [C.c_double] * 5 + [_dp, C.c_int]
        f("polar").restype = C.c_double
        f("hexadecapole").argtypes = [st] + [C.c_double] * 5 + [_dp, _dp]
        f("caustic_cache").argtypes = [C.c_double, C.c_double, C.c_int, _dp, C.c_int, _dp, _dp]
        f("caustic_distances").argtypes = [C.c_double] * 2 + [C.c_int] + [C.c_double] * 3 + [_dp]
        f("critical_sources").argtypes = [C.c_double] * 3 + [_dp]
        f("ld_brightness").argtypes = [C.c_double] * 3
        f("ld_brightness").restype = C.c_double
        f("light_curve_static").argtypes = [st, _dp, C.c_int] + [C.c_double] * 7 + [_dp, _ip]

    def binary_mag(self, st, s, q, x, y, rho, a_ps, ps_exact=True):
        d = np.zeros(2)
        i = np.zeros(4, dtype=np.int32)
        self.fn("binary_mag")(C.byref(st), s, q, x, y, rho, a_ps, int(ps_exact), _ptr(d), _ptr(i, _ip))
        return dict(A=d[0], err=d[1], method=int(i[0]), level=int(i[1]), converged=bool(i[2]))

    def inverse_ray(self, st, s, q, x, y, rho):
        s, q, x, y, rho = (_f64(np.broadcast_to(v, np.broadcast(s, q, x, y, rho).shape)).ravel()
                           for v in (s, q, x, y, rho))
        n = s.size
        A = np.empty(n)
        m = np.empty(n, dtype=np.int32)
        self.fn("inverse_ray_many")(C.byref(st), n, _ptr(s), _ptr(q), _ptr(x), _ptr(y), _ptr(rho),
                                    _ptr(A), _ptr(m, _ip))
        return A, m

    def inverse_ray_fixed(self, st, s, q, x, y, rho):
        """inverse_ray plus, for polar points, the integral with its cells summed
        exactly the device's way (a 128-bit fixed-point sum) and the cell count."""
        s, q, x, y, rho = (_f64(np.broadcast_to(v, np.broadcast(s, q, x, y, rho).shape)).ravel()
                           for v in (s, q, x, y, rho))
        n = s.size
        A = np.empty(n)
        m = np.empty(n, dtype=np.int32)
        Af = np.empty(n)
        cells = np.zeros(n, dtype=np.uint64)
        self.fn("inverse_ray_many_fixed")(C.byref(st), n, _ptr(s), _ptr(q), _ptr(x), _ptr(y), _ptr(rho),
                                          _ptr(A), _ptr(m, _ip), _ptr(Af), cells.ctypes.data)
        return A, m, Af, cells

    def seeds(self, st, s, q, x, y, rho, cap=512):
        out = np.zeros(2 * cap)
        n = self.fn("seeds")(C.byref(st), s, q, x, y, rho, _ptr(out), cap)
        return out[: 2 * min(n, cap)].reshape(-1, 2)

    def cartesian(self, st, s, q, x, y, rho, seeds):
        sd = _f64(seeds).ravel()
        diag = np.zeros(8)
        A = self.fn("cartesian")(C.byref(st), s, q, x, y, rho, _ptr(sd), sd.size // 2, _ptr(diag))
        return A, diag

    def polar(self, st, s, q, x, y, rho, seeds):
        sd = _f64(seeds).ravel()
        return self.fn("polar")(C.byref(st), s, q, x, y, rho, _ptr(sd), sd.size // 2)

    def hexadecapole(self, st, s, q, x, y, rho, a0=None):
        out = np.zeros(2)
        k = None if a0 is None else C.byref(C.c_double(a0))
        self.fn("hexadecapole")(C.byref(st), s, q, x, y, rho, k, _ptr(out))
        return out[0], out[1]

    def caustic_cache(self, s, q, bins=1400):
        cap = max(bins, 32)
        br = np.zeros(4 * cap * 2)
        bbox = np.zeros(4)
        ms = C.c_double()
        per = self.fn("caustic_cache")(s, q, bins, _ptr(br), cap, _ptr(bbox), C.byref(ms))
        return br.reshape(4, cap, 2)[:, :per], bbox, ms.value

    def caustic_distances(self, s, q, x, y, search_radius, bins=1400):
        out = np.zeros(2)
        self.fn("caustic_distances")(s, q, bins, x, y, search_radius, _ptr(out))
        return out[0], out[1]

    def critical_sources(self, s, q, phi):
        out = np.zeros(8)
        n = self.fn("critical_sources")(s, q, phi, _ptr(out))
        return out[: 2 * n].reshape(-1, 2)

    def ld_brightness(self, c, d, r2):
        return self.fn("ld_brightness")(c, d, r2)

    def light_curve_static(self, st, times, t0, tE, u0, alpha, s, q, rho):
        t = _f64(times)
        out = np.empty(t.size)
        m = np.empty(t.size, dtype=np.int32)
        rc = self.fn("light_curve_static")(C.byref(st), _ptr(t), t.size, t0, tE, u0, alpha, s, q, rho,
                                           _ptr(out), _ptr(m, _ip))
        return out, m, rc


class Oracle(_FsLib):
    """The CPU restatement."""

    def __init__(self):
        super().__init__(ORACLE_SO, "orc_")


class Reference(_FsLib):
    """The reference compiled from its own sources (oracle/_ref)."""

    def __init__(self):
        super().__init__(REF_SO, "ref_")


def import_reference_module():
    """The reference's own pybind11 module (oracle/_ref/lcbinint*.so), or None."""
    import importlib.util
    import sys
    for f in REF_DIR.glob("lcbinint*.so"):
        spec = importlib.util.spec_from_file_location("lcbinint", f)
        mod = importlib.util.module_from_spec(spec)
        sys.modules.setdefault("lcbinint_reference", mod)
        spec.loader.exec_module(mod)
        return mod
    return None


def have_reference() -> bool:
    return REF_SO.exists()
