"""Python mirror of the reference's pybind11 API for the magnification path.

Names, argument names, defaults and error behaviour follow
python/lcbinint_pybind.cpp (Options :2985-3112, LimbDarkening :2828-2846,
LightCurve :3114-3406, binary_mag0 :3819-3824, binary_inverse_ray :3826-3847).
Every computation is a call into the C ABI of the CUDA library.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import context


class LcbiStructs:
    class FsSettings(C.Structure):
        _fields_ = [
            ("source_bins", C.c_int32), ("caustic_bins", C.c_int32), ("grid_ratio", C.c_double),
            ("polar_source_bins", C.c_int32), ("polar_grid_ratio", C.c_double), ("finite_mode", C.c_int32),
            ("kinji_threshold", C.c_double), ("hex_threshold", C.c_double),
            ("adaptive_hex_threshold", C.c_double), ("limb_darkening_c", C.c_double),
            ("limb_darkening_d", C.c_double), ("adaptive_source_bins", C.c_int32),
            ("max_source_bins", C.c_int32), ("finite_source_tol", C.c_double),
            ("finite_source_reltol", C.c_double),
        ]

    class FsPoint(C.Structure):
        _fields_ = [("s", C.c_double), ("q", C.c_double), ("y1", C.c_double), ("y2", C.c_double),
                    ("rho", C.c_double), ("point_source_magnification", C.c_double),
                    ("settings", C.c_int32), ("model", C.c_int32), ("flags", C.c_int32),
                    ("reserved", C.c_int32)]

    class FsResult(C.Structure):
        _fields_ = [("magnification", C.c_double), ("error_estimate", C.c_double), ("method", C.c_int32),
                    ("converged", C.c_int32), ("status", C.c_int32), ("seed_count", C.c_int32)]


FS_POINT_DTYPE = np.dtype([("s", "f8"), ("q", "f8"), ("y1", "f8"), ("y2", "f8"), ("rho", "f8"),
                           ("a_ps", "f8"), ("settings", "i4"), ("model", "i4"), ("flags", "i4"),
                           ("reserved", "i4")])
FS_RESULT_DTYPE = np.dtype([("magnification", "f8"), ("error_estimate", "f8"), ("method", "i4"),
                            ("converged", "i4"), ("status", "i4"), ("seed_count", "i4")])
PS_EXACT = 1
PS_ON_DEVICE = 2
METHOD_NAMES = {0: "point_source", 1: "hexadecapole", 2: "inverse_ray_cartesian", 3: "inverse_ray_polar",
                4: "inverse_ray_spine", 5: "source_plane_quadrature"}


@dataclass
class LimbDarkening:
    """Source surface brightness I = 1 - c(1 - mu) - d(1 - sqrt(mu)) (PYB:2828-2846)."""

    c: float = 0.0
    d: float = 0.0

    @staticmethod
    def none() -> "LimbDarkening":
        return LimbDarkening()

    @staticmethod
    def linear(c: float) -> "LimbDarkening":
        return LimbDarkening(float(c), 0.0)

    @staticmethod
    def quadratic(c: float, d: float) -> "LimbDarkening":
        return LimbDarkening(float(c), float(d))

    def __repr__(self):
        return f"LimbDarkening(c={self.c:.6f}, d={self.d:.6f})"


@dataclass
class EventCoordinates:
    ra: float = 0.0
    dec: float = 0.0
    tfix: float = 0.0
    obs_lat: float = 0.0
    obs_lon: float = 0.0


_GRID_MODE = {"auto": 4, "": 4, "cartesian": 1, "inverse_ray_cartesian": 1, "polar": 2, "inverse_ray_polar": 2}
_GRID_NAME = {4: "auto", 1: "cartesian", 2: "polar"}


def _apply_param_type(o: "Options", name: str):
    # apply_param_type (PYB:246-276)
    if name in ("auto", "", "vbm", "vbbl", "standard"):
        o.center_of_mass, o.vbm_compatible = 0, 1
    elif name in ("lcbinint", "original", "legacy"):
        o.center_of_mass, o.vbm_compatible = 0, 0
    elif name == "center_of_mass":
        o.center_of_mass, o.vbm_compatible = 1, 0
    elif name == "vbm_center_of_mass":
        o.center_of_mass, o.vbm_compatible = 1, 1
    else:
        raise ValueError("param_type must be 'vbm', 'lcbinint', 'original', or 'center_of_mass'")


_XALLARAP_TYPE = {"": 0, "none": 0, "angular_velocity": 1, "orbital_elements": 2}


class Options:
    """Computation options; defaults and aliases of lcbinint.Options (PYB:2985-3112)."""

    def __init__(self, source_bins: int = 50, nbin=None, inverse_ray_grid: str = "auto",
                 caustic_bins: int = 1400, grid_ratio: float = 4.0, polar_nbin=None, polar_source_bins=None,
                 polar_grid_ratio=None, point_source_threshold: float = 20.0,
                 hexadecapole_threshold: float = 3.0, adaptive_hex_threshold: float = 0.001,
                 adaptive_source_bins: int = -1, max_source_bins: int = 400, finite_source_tol: float = 0.0,
                 finite_source_reltol: float = 0.0, tol: float = math.nan, reltol: float = math.nan,
                 coordinates: str = "auto", hex_tol: float = math.nan, param_type: str = "auto",
                 xallarap_param_type: str = "none"):
        self.center_of_mass, self.vbm_compatible = 0, 1
        if param_type and param_type != "auto":
            _apply_param_type(self, param_type)
        else:
            _apply_param_type(self, coordinates)
        if xallarap_param_type not in ("", "none", "angular_velocity", "orbital_elements"):
            raise ValueError("xallarap_param_type must be 'none', 'angular_velocity', or 'orbital_elements'")
        self._xallarap = xallarap_param_type or "none"
        self.inverse_ray_grid = inverse_ray_grid
        self.source_bins = int(source_bins if nbin is None else nbin)
        self.caustic_bins = int(caustic_bins)
        self.grid_ratio = float(grid_ratio)
        pn = polar_nbin if polar_nbin is not None else polar_source_bins
        self.polar_source_bins = int(pn) if pn is not None else 0
        self._polar_grid_ratio = float(polar_grid_ratio) if polar_grid_ratio is not None else 0.0
        self.point_source_threshold = float(point_source_threshold)
        self.hexadecapole_threshold = float(hexadecapole_threshold)
        self.adaptive_hex_threshold = float(adaptive_hex_threshold if math.isnan(hex_tol) else hex_tol)
        self.max_source_bins = int(max_source_bins)
        self.finite_source_tol = float(finite_source_tol if math.isnan(tol) else tol)
        self.finite_source_reltol = float(finite_source_reltol if math.isnan(reltol) else reltol)
        self.adaptive_source_bins = 0 if adaptive_source_bins < 0 else int(adaptive_source_bins)

    # ---- properties with the reference's aliases ----
    @property
    def nbin(self) -> int:
        return self.source_bins

    @nbin.setter
    def nbin(self, v: int):
        self.source_bins = int(v)

    @property
    def inverse_ray_grid(self) -> str:
        return _GRID_NAME.get(self._mode, "internal")

    @inverse_ray_grid.setter
    def inverse_ray_grid(self, v: str):
        if v not in _GRID_MODE:
            raise ValueError("inverse_ray_grid must be 'auto', 'cartesian', or 'polar'")
        self._mode = _GRID_MODE[v]

    @property
    def polar_nbin(self):
        return self.polar_source_bins if self.polar_source_bins > 0 else None

    @polar_nbin.setter
    def polar_nbin(self, v):
        self.polar_source_bins = 0 if v is None else int(v)

    @property
    def polar_grid_ratio(self):
        return self._polar_grid_ratio if self._polar_grid_ratio > 0 else None

    @polar_grid_ratio.setter
    def polar_grid_ratio(self, v):
        self._polar_grid_ratio = 0.0 if v is None else float(v)

    @property
    def hex_tol(self) -> float:
        return self.adaptive_hex_threshold

    @hex_tol.setter
    def hex_tol(self, v):
        self.adaptive_hex_threshold = float(v)

    @property
    def tol(self) -> float:
        return self.finite_source_tol

    @tol.setter
    def tol(self, v):
        self.finite_source_tol = float(v)

    @property
    def reltol(self) -> float:
        return self.finite_source_reltol

    @reltol.setter
    def reltol(self, v):
        self.finite_source_reltol = float(v)

    @property
    def coordinates(self) -> str:
        if self.vbm_compatible and not self.center_of_mass:
            return "vbm"
        if self.center_of_mass and self.vbm_compatible:
            return "vbm_center_of_mass"
        if self.center_of_mass:
            return "center_of_mass"
        return "lcbinint"

    @coordinates.setter
    def coordinates(self, v: str):
        _apply_param_type(self, v)

    param_type = coordinates

    @property
    def xallarap_param_type(self) -> str:
        return self._xallarap

    def c_options(self) -> np.ndarray:
        """The lcbi_options this Options stands for (PYB:2985-3037 on top of
        public_default_options, PYB:213-220), as a one-element array."""
        o = _lib.default_options()
        o["center_of_mass"] = self.center_of_mass
        o["vbm_compatible"] = self.vbm_compatible
        o["mode"] = self._mode
        o["xallarap_param_type"] = _XALLARAP_TYPE[self._xallarap]
        o["source_bins"] = self.source_bins
        o["caustic_bins"] = self.caustic_bins
        o["grid_ratio"] = self.grid_ratio
        o["polar_source_bins"] = self.polar_source_bins
        o["polar_grid_ratio"] = self._polar_grid_ratio
        o["point_source_threshold"] = self.point_source_threshold
        o["hexadecapole_threshold"] = self.hexadecapole_threshold
        o["adaptive_hex_threshold"] = self.adaptive_hex_threshold
        o["adaptive_source_bins"] = self.adaptive_source_bins
        o["max_source_bins"] = self.max_source_bins
        o["finite_source_tol"] = self.finite_source_tol
        o["finite_source_reltol"] = self.finite_source_reltol
        return o

    def fs_settings(self, ld: LimbDarkening) -> LcbiStructs.FsSettings:
        """make_finite_source_settings (PYB:471-492)."""
        return LcbiStructs.FsSettings(
            source_bins=self.source_bins, caustic_bins=self.caustic_bins, grid_ratio=self.grid_ratio,
            polar_source_bins=self.polar_source_bins, polar_grid_ratio=self._polar_grid_ratio,
            finite_mode=self._mode, kinji_threshold=self.point_source_threshold,
            hex_threshold=self.hexadecapole_threshold, adaptive_hex_threshold=self.adaptive_hex_threshold,
            limb_darkening_c=ld.c, limb_darkening_d=ld.d, adaptive_source_bins=self.adaptive_source_bins,
            max_source_bins=self.max_source_bins, finite_source_tol=self.finite_source_tol,
            finite_source_reltol=self.finite_source_reltol)


def _raise_for_status(status, what="numerical error"):
    status = np.asarray(status)
    bad = status != _lib.LCBI_OK
    if bad.any():
        code = int(status[bad][0])
        if code == _lib.LCBI_NUMERICAL_ERROR:
            raise RuntimeError("numerical error")
        if code == _lib.LCBI_UNSUPPORTED:
            raise RuntimeError("unsupported")
        raise RuntimeError(f"{what}: device limit reached (status {code})")


def binary_mag(points, settings_list, *, device: int = 0, models=None):
    """Batched FiniteSourceMagnifier::binary_mag over a structured array of
    FS_POINT_DTYPE records; returns a FS_RESULT_DTYPE array."""
    pts = np.ascontiguousarray(points, dtype=FS_POINT_DTYPE)
    n = pts.size
    res = np.zeros(n, dtype=FS_RESULT_DTYPE)
    if n == 0:
        return res
    st = (LcbiStructs.FsSettings * len(settings_list))(*settings_list)
    ctx = context(device)
    flags = 0
    mptr, nm = None, 0
    if models is not None:
        md = np.ascontiguousarray(models, dtype=np.dtype([("s", "f8"), ("q", "f8"), ("bins", "i4"),
                                                             ("r", "i4")]))
        mptr, nm = md.ctypes.data, md.size
        flags |= 2
    rc = ctx._L.lcbi_gpu_binary_mag(ctx.handle, st, len(settings_list), mptr, nm, n, pts.ctypes.data,
                                    res.ctypes.data, flags)
    ctx.check(rc, "lcbi_gpu_binary_mag")
    return res


def binary_inverse_ray_batch(s, q, x, y, rho, limb_darkening: LimbDarkening = None, options: Options = None,
                             *, device: int = 0, return_method: bool = False):
    """Batched lcbinint.binary_inverse_ray: the same forced inverse-ray decision
    per point (PYB:3826-3847), all points in one launch sequence."""
    ld = limb_darkening or LimbDarkening()
    opt = options or Options()
    arrs = np.broadcast_arrays(s, q, x, y, rho)
    shape = arrs[0].shape
    s, q, x, y, rho = (_lib.as_f64(a) for a in arrs)
    n = s.size
    A = np.empty(n)
    method = np.empty(n, dtype=np.int32)
    status = np.empty(n, dtype=np.int32)
    st = opt.fs_settings(ld)
    ctx = context(device)
    rc = ctx._L.lcbi_gpu_binary_inverse_ray(ctx.handle, C.byref(st), n, _lib.ptr(s), _lib.ptr(q), _lib.ptr(x),
                                            _lib.ptr(y), _lib.ptr(rho), _lib.ptr(A), _lib.ptr(method),
                                            _lib.ptr(status))
    ctx.check(rc, "lcbi_gpu_binary_inverse_ray")
    if return_method:
        return A.reshape(shape), method.reshape(shape), status.reshape(shape)
    return A.reshape(shape)


def binary_inverse_ray(s: float, q: float, x: float, y: float, rho: float,
                       limb_darkening: LimbDarkening = None, options: Options = None) -> float:
    """Binary finite-source magnification at (x, y) by inverse-ray shooting,
    same convention as VBMicrolensing BinaryMag2 (PYB:3826-3847)."""
    return float(binary_inverse_ray_batch(s, q, x, y, rho, limb_darkening, options).reshape(-1)[0])


def light_curves(times_list, params_list, options: Options = None, limb_darkening: LimbDarkening = None,
                 *, device: int = 0, return_method: bool = False):
    """Many static binary light curves (VBM convention) in one batched launch.

    times_list[m] are model m's epochs; params_list[m] is a dict with t0, tE,
    u0, alpha, s, q, rho.  Returns a list of arrays."""
    opt = options or Options()
    ld = limb_darkening or LimbDarkening()
    nm = len(params_list)
    counts = np.array([len(t) for t in times_list], dtype=np.int32)
    first = np.zeros(nm, dtype=np.int64)
    if nm > 1:
        first[1:] = np.cumsum(counts[:-1])
    times = np.ascontiguousarray(np.concatenate([np.asarray(t, dtype=np.float64).ravel() for t in times_list])
                                 if nm else np.zeros(0))
    P = np.array([[p.get("t0", 0.0), p.get("tE", 1.0), p.get("u0", 0.0), p.get("alpha", 0.0),
                   p.get("s", 1.0), p.get("q", 1.0), p.get("rho", 0.0)] for p in params_list],
                 dtype=np.float64).reshape(nm, 7)
    n = times.size
    A = np.empty(n)
    method = np.empty(n, dtype=np.int32)
    status = np.empty(n, dtype=np.int32)
    st = opt.fs_settings(ld)
    ctx = context(device)
    rc = ctx._L.lcbi_gpu_light_curves(ctx.handle, C.byref(st), nm, _lib.ptr(P), _lib.ptr(first), _lib.ptr(counts),
                                      _lib.ptr(times), n, _lib.ptr(A), _lib.ptr(method), _lib.ptr(status))
    ctx.check(rc, "lcbi_gpu_light_curves")
    out = np.split(A, np.cumsum(counts)[:-1]) if nm else []
    if return_method:
        return out, np.split(method, np.cumsum(counts)[:-1]), np.split(status, np.cumsum(counts)[:-1])
    return out


STATIC = 0
CIRCULAR = 1
KEPLER = 2


def set_earth_ephemeris(path) -> int:
    """Loads the Earth ephemeris for annual parallax (a JPL Horizons vector
    table) instead of the file named by LCBININT_EARTH_EPHEMERIS; returns the
    number of states read (lcbi_set_earth_ephemeris)."""
    n = _lib.lib().lcbi_set_earth_ephemeris(str(path).encode())
    if n < 0:
        raise FileNotFoundError(str(path))
    return n


def circular_orbital_motion(time, separation, angle, g1=0.0, g2=0.0, g3=0.0, reference_time=0.0):
    """lcbinint.circular_orbital_motion (PYB:3896-3908): (separation, angle,
    line-of-sight separation) of a circular lens orbit at `time`."""
    out = np.zeros(3)
    _lib.lib().lcbi_circular_orbital_motion(float(time), float(separation), float(angle), float(g1), float(g2),
                                            float(g3), float(reference_time), _lib.ptr(out))
    return float(out[0]), float(out[1]), float(out[2])


def kepler_orbital_motion(time, separation, angle, g1=0.0, g2=0.0, g3=0.0, szs=0.0, ar=1.0, reference_time=0.0):
    """lcbinint.kepler_orbital_motion (PYB:3910-3925): the Keplerian counterpart."""
    out = np.zeros(3)
    _lib.lib().lcbi_kepler_orbital_motion(float(time), float(separation), float(angle), float(g1), float(g2),
                                          float(g3), float(szs), float(ar), float(reference_time), _lib.ptr(out))
    return float(out[0]), float(out[1]), float(out[2])


@dataclass
class GeometryBranches:
    """lcbinint.GeometryBranches (PYB:51-54, 2811-2813): four tracked branches."""
    x: list = field(default_factory=list)
    y: list = field(default_factory=list)


@dataclass
class GeometryCurve:
    """lcbinint.GeometryCurve (PYB:45-49, 2806-2809): a source trajectory."""
    times: list = field(default_factory=list)
    x: list = field(default_factory=list)
    y: list = field(default_factory=list)


def binary_geometry(s: float, q_core: float, n_points: int, caustic: bool, *, device: int = 0) -> GeometryBranches:
    """Caustic or critical-curve branches of a binary lens (lcbi_gpu_binary_geometry)."""
    if int(n_points) < 8:
        raise ValueError("n_points must be at least 8")
    n = int(n_points)
    xy = np.empty((4, n, 2))
    ctx = context(device)
    rc = ctx._L.lcbi_gpu_binary_geometry(ctx.handle, float(s), float(q_core), n, 1 if caustic else 0,
                                         _lib.ptr(xy), None)
    ctx.check(rc, "lcbi_gpu_binary_geometry")
    return GeometryBranches([xy[b, :, 0].tolist() for b in range(4)], [xy[b, :, 1].tolist() for b in range(4)])

# Parameter-dictionary keys and defaults (PyBinaryParams, PYB:103-134).
_BINARY_PARAM_DEFAULTS = dict(t0=0.0, tE=1.0, u0=0.0, alpha=0.0, s=1.0, q=1.0, q2=0.0, sep2=0.0, ang=0.0, rho=0.0,
                              piEN=0.0, piEE=0.0, g1=0.0, g2=0.0, g3=0.0, lom_szs=0.0, lom_ar=1.0, u0_2=0.0,
                              t0_2=0.0, flux_ratio=0.0, xi_1=0.0, xi_2=0.0, omega_xa=0.0, inc_xa=0.0, phi_xa=0.0,
                              piEN_xa=0.0, piEE_xa=0.0, period_xa=0.0, ecc_xa=0.0, peri_xa=0.0)


def binary_c_params(params_list, limb_darkening: LimbDarkening = None, event: EventCoordinates = None,
                    orbital_motion_mode: int = STATIC, parallax: bool = False,
                    terrestrial_parallax: bool = False) -> np.ndarray:
    """lcbi_params of single-source binary-lens parameter dictionaries, as
    make_c_params_for_single_source builds them (PYB:2721-2748, with
    make_binary_params PYB:338-401): the parallax components count only with
    parallax, the observatory only with terrestrial parallax."""
    ld = limb_darkening or LimbDarkening()
    ev = event or EventCoordinates()
    out = _lib.default_params(len(params_list))
    for i, d in enumerate(params_list):
        p = dict(_BINARY_PARAM_DEFAULTS)
        p.update(d)
        r = out[i]
        r["t0"], r["tE"], r["umin"], r["theta"] = p["t0"], p["tE"], p["u0"], p["alpha"]
        r["sep"], r["q"], r["rho"] = p["s"], p["q"], p["rho"]
        r["limb_darkening_c"], r["limb_darkening_d"] = ld.c, ld.d
        r["ra"], r["dec"], r["tfix"] = ev.ra, ev.dec, ev.tfix
        if terrestrial_parallax:
            r["obs_lat"], r["obs_lon"] = ev.obs_lat, ev.obs_lon
        if parallax:
            r["piEN"], r["piEE"] = p["piEN"], p["piEE"]
        r["g1"], r["g2"], r["g3"] = p["g1"], p["g2"], p["g3"]
        r["orbital_motion_mode"] = int(orbital_motion_mode)
        r["lom_szs"], r["lom_ar"] = p["lom_szs"], p["lom_ar"]
        for k in ("xi_1", "xi_2", "omega_xa", "inc_xa", "phi_xa", "piEN_xa", "piEE_xa", "period_xa", "ecc_xa",
                  "peri_xa"):
            r[k] = p[k]
    return out


def magnification_arrays(times_list, c_params: np.ndarray, options: Options = None, *, keyword_route: bool = False,
                         device: int = 0):
    """lcbi_magnification_array for many parameter sets in one batched GPU
    pass (lcbi_gpu_magnification_arrays).  c_params is an array of
    PARAMS_DTYPE records (binary_c_params builds them from dictionaries).
    Returns (results, status): per set an array of RESULT_DTYPE records and
    the status lcbi_magnification_array would have returned."""
    opt = options or Options()
    c_params = np.ascontiguousarray(c_params, dtype=_lib.PARAMS_DTYPE)
    nm = len(c_params)
    counts = np.array([len(t) for t in times_list], dtype=np.int32)
    first = np.zeros(nm, dtype=np.int64)
    if nm > 1:
        first[1:] = np.cumsum(counts[:-1])
    times = np.ascontiguousarray(np.concatenate([np.asarray(t, dtype=np.float64).ravel() for t in times_list])
                                 if nm else np.zeros(0))
    res = np.zeros(times.size, dtype=_lib.RESULT_DTYPE)
    status = np.zeros(nm, dtype=np.int32)
    if nm == 0:
        return [], status
    co = opt.c_options()
    ctx = context(device)
    rc = ctx._L.lcbi_gpu_magnification_arrays(ctx.handle, nm, _lib.ptr(c_params), _lib.ptr(co), _lib.ptr(first),
                                              _lib.ptr(counts), _lib.ptr(times), times.size,
                                              _lib.ARRAYS_KEYWORD_ROUTE if keyword_route else 0, _lib.ptr(res),
                                              _lib.ptr(status))
    ctx.check(rc, "lcbi_gpu_magnification_arrays")
    return np.split(res, np.cumsum(counts)[:-1]), status


def _raise_for_c_status(status):
    # direct_dynamic_fill_values / evaluate_binary_light_curve_numpy (PYB:1074-1083, 1160-1171)
    for st in np.asarray(status).ravel():
        if st == _lib.LCBI_UNSUPPORTED:
            raise RuntimeError("unsupported")
        if st == _lib.LCBI_INVALID_ARGUMENT:
            raise ValueError("invalid argument")
        if st != _lib.LCBI_OK:
            raise RuntimeError("numerical error")


class LightCurve:
    """lcbinint.LightCurve (PYB:3114-3406): a reusable light-curve callable.

    Routes as the reference does.  The static binary lens in VBM coordinates
    takes the direct fast path (PYB:1087-1174, lcbi_gpu_light_curves).  Lens
    orbital motion (circular or Keplerian), annual and terrestrial parallax
    (with an Earth ephemeris: set_earth_ephemeris or the
    LCBININT_EARTH_EPHEMERIS environment variable), xallarap and the
    original / centre-of-mass conventions take LensModel's path when the
    parameters come as a dictionary (PYB:2325-2358 -> lens_model.cpp) and the
    dynamic path when they come as keywords (PYB:1364-1385, 1958-2060); both
    run through lcbi_gpu_magnification_arrays.  Binary sources blend two
    single-source curves (PYB:2331-2354).  Triple lenses are outside this
    implementation and raise NotImplementedError."""

    _KEYWORDS = ("t0", "tE", "u0", "alpha", "s", "q", "rho", "piEN", "piEE", "g1", "g2", "g3", "lom_szs", "lom_ar")

    def __init__(self, *, lens: str = "binary_lens", source: str = "single", event: EventCoordinates = None,
                 options: Options = None, limb_darkening: LimbDarkening = None, orbital_motion_mode: int = STATIC,
                 parallax: bool = False, terrestrial_parallax: bool = False):
        if lens not in ("binary_lens", "binary", "binary-lens", ""):
            if lens in ("triple_lens", "triple"):
                raise NotImplementedError("triple lenses are outside this implementation")
            raise ValueError("lens must be 'binary_lens' or 'triple_lens'")
        if source in ("", "single"):
            source = "single"
        elif source in ("binary", "binary_source"):
            source = "binary"
        else:
            raise ValueError("source must be 'single' or 'binary'")
        self.lens = "binary_lens"
        self.source = source
        self.event = event or EventCoordinates()
        self.options = options or Options()
        self.limb_darkening = limb_darkening or LimbDarkening()
        self.orbital_motion_mode = int(orbital_motion_mode)
        if self.orbital_motion_mode not in (STATIC, CIRCULAR, KEPLER):
            raise ValueError("orbital_motion_mode must be STATIC, CIRCULAR or KEPLER")
        self.parallax = parallax
        self.terrestrial_parallax = terrestrial_parallax

    def _direct(self, p=None, keyword_route=False) -> bool:
        # can_use_direct_static_binary (PYB:494-503); for dictionaries also
        # evaluate_binary_light_curve_numpy's test (PYB:1105-1118).
        o = self.options
        if not (self.orbital_motion_mode == STATIC and o.vbm_compatible and not o.center_of_mass):
            return False
        if keyword_route:
            # The keyword overloads take the dynamic path whenever the curve
            # has parallax (PYB:2360-2405).
            return not self.parallax
        keys = ("xi_1", "xi_2", "piEN_xa", "piEE_xa") + (("piEN", "piEE") if self.parallax else ())
        return all(p.get(k, 0.0) == 0.0 for k in keys)

    def _single(self, times, p, keyword_route=False):
        if self._direct(p, keyword_route):
            (A,), (m,), (st,) = light_curves([times], [p], self.options, self.limb_darkening, return_method=True)
            _raise_for_status(st)
            return A
        if keyword_route:
            # PyLightCurveFunc::dynamic_light_curve (PYB:1364-1385): parallax
            # components as given, the observatory from the event coordinates.
            cp = binary_c_params([p], self.limb_darkening, self.event, self.orbital_motion_mode, parallax=True,
                                 terrestrial_parallax=True)
        else:
            cp = binary_c_params([p], self.limb_darkening, self.event, self.orbital_motion_mode,
                                 parallax=self.parallax, terrestrial_parallax=self.terrestrial_parallax)
        (res,), status = magnification_arrays([times], cp, self.options, keyword_route=keyword_route)
        _raise_for_c_status(status)
        return res["magnification"].copy()

    def __call__(self, times, params=None, **kw):
        times = np.ascontiguousarray(times, dtype=np.float64)
        if times.ndim != 1:
            raise ValueError("times must be one-dimensional")
        if params is not None:
            if kw:
                raise TypeError("pass the parameters either as a dictionary or as keywords")
            p = dict(params)
            keyword_route = False
        else:
            unknown = set(kw) - set(self._KEYWORDS)
            if unknown:
                raise TypeError(f"unexpected keyword arguments: {sorted(unknown)}")
            if ("piEN" in kw or "piEE" in kw) and not self.parallax:
                raise ValueError("piEN/piEE require LightCurve(parallax=True); the current trajectory model is static")
            p = dict(kw)
            keyword_route = True
        if self.source == "binary":
            p2 = dict(p)
            p2["u0"] = p.get("u0_2", 0.0)
            p2["t0"] = p.get("t0_2", 0.0)
            v1 = self._single(times, p)
            v2 = self._single(times, p2)
            fr = p.get("flux_ratio", 0.0)
            inv = 1.0 / (1.0 + fr)
            return (v1 + fr * v2) * inv
        return self._single(times, p, keyword_route)

    light_curve = __call__

    def list(self, times, **kw):
        return [float(v) for v in self(np.asarray(times, dtype=np.float64), **kw)]

    def magnification(self, time, params=None, **kw):
        return float(self(np.array([float(time)]), params, **kw)[0])

    _GEOMETRY_KEYWORDS = dict(s=1.0, q=1.0, n_points=1400, time=math.nan, t0=0.0, tE=1.0, u0=0.0, alpha=0.0,
                              g1=0.0, g2=0.0, g3=0.0, lom_szs=0.0, lom_ar=1.0)

    def _geometry(self, caustic, params, n_points, kw):
        # caustics_from_dict (PYB:2539-2556) and geometry_branches (PYB:1882-1926).
        if params is not None:
            if kw:
                raise TypeError("pass the parameters either as a dictionary or as keywords")
            p = dict(_BINARY_PARAM_DEFAULTS)
            p.update(params)
            g = dict(self._GEOMETRY_KEYWORDS, s=p["s"], q=p["q"], n_points=1000 if n_points is None else n_points)
        else:
            unknown = set(kw) - set(self._GEOMETRY_KEYWORDS)
            if unknown:
                raise TypeError(f"unexpected keyword arguments: {sorted(unknown)}")
            g = dict(self._GEOMETRY_KEYWORDS)
            g.update(kw)
            if n_points is not None:
                g["n_points"] = n_points
        if int(g["n_points"]) < 8:
            raise ValueError("n_points must be at least 8")
        separation = g["s"]
        if self.orbital_motion_mode != STATIC and math.isfinite(g["time"]):
            t_ref = self.event.tfix if self.event.tfix != 0.0 else g["t0"]
            if self.orbital_motion_mode == CIRCULAR:
                separation = circular_orbital_motion(g["time"], g["s"], g["alpha"], g["g1"], g["g2"], g["g3"],
                                                     t_ref)[0]
            else:
                separation = kepler_orbital_motion(g["time"], g["s"], g["alpha"], g["g1"], g["g2"], g["g3"],
                                                   g["lom_szs"], g["lom_ar"], t_ref)[0]
        q = g["q"]
        q_core = 1.0 / q if (self.options.vbm_compatible and q != 0.0) else q
        return binary_geometry(separation, q_core, int(g["n_points"]), caustic)

    _TRAJECTORY_KEYWORDS = ("t0", "tE", "u0", "alpha", "s", "q", "piEN", "piEE", "g1", "g2", "g3", "lom_szs",
                            "lom_ar")

    def source_trajectory(self, times, params=None, **kw) -> GeometryCurve:
        """LightCurve.source_trajectory (PYB:3292-3330): the source position in the
        lens frame at each time (lcbi_source_trajectory).  A dictionary's
        piEN/piEE always count (PYB:2529-2537); as keywords they need
        LightCurve(parallax=True) (PYB:2580-2600)."""
        times = np.ascontiguousarray(times, dtype=np.float64).ravel()
        if params is not None:
            if kw:
                raise TypeError("pass the parameters either as a dictionary or as keywords")
            p = dict(params)
        else:
            unknown = set(kw) - set(self._TRAJECTORY_KEYWORDS)
            if unknown:
                raise TypeError(f"unexpected keyword arguments: {sorted(unknown)}")
            if ("piEN" in kw or "piEE" in kw) and not self.parallax:
                raise ValueError("piEN/piEE require LightCurve(parallax=True); the current trajectory model is static")
            p = dict(kw)
        p["rho"] = 0.0
        cp = binary_c_params([p], self.limb_darkening, self.event, self.orbital_motion_mode, parallax=True,
                             terrestrial_parallax=True)
        co = self.options.c_options()
        x = np.empty(times.size)
        y = np.empty(times.size)
        L = _lib.lib()
        rc = L.lcbi_source_trajectory(_lib.ptr(cp), _lib.ptr(co), _lib.ptr(times), times.size, _lib.ptr(x),
                                      _lib.ptr(y))
        if rc != _lib.LCBI_OK:
            raise ValueError("invalid argument")
        return GeometryCurve(times=times.tolist(), x=x.tolist(), y=y.tolist())

    def caustics(self, params=None, n_points=None, **kw):
        """LightCurve.caustics (PYB:1525-1542, 2539-2556): four tracked caustic branches."""
        return self._geometry(True, params, n_points, kw)

    def critical_curves(self, params=None, n_points=None, **kw):
        """LightCurve.critical_curves (PYB:1544-1561): four tracked critical-curve branches."""
        return self._geometry(False, params, n_points, kw)

    def info(self, times, params=None, **kw):
        """Per-epoch magnifications with the finite-source method chosen."""
        times = np.ascontiguousarray(times, dtype=np.float64)
        p = dict(params) if params is not None else {}
        p.update(kw)
        if not self._direct(p):
            raise NotImplementedError("info() is implemented for the static binary lens in VBM coordinates")
        (A,), (m,), (st,) = light_curves([times], [p], self.options, self.limb_darkening, return_method=True)
        _raise_for_status(st)
        return LightCurveInfo(times=list(times), magnifications=list(A), finite_source_methods=list(m),
                              finite_source_method_names=[METHOD_NAMES[int(v)] for v in m])


@dataclass
class LightCurveInfo:
    times: list = field(default_factory=list)
    magnifications: list = field(default_factory=list)
    finite_source_methods: list = field(default_factory=list)
    finite_source_method_names: list = field(default_factory=list)


LightCurveFunc = LightCurve
