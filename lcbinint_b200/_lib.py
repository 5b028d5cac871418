"""ctypes binding of the in-tree CUDA library (liblcbinint_b200.so).

The library is the product: there is no CPU fallback.  Loading fails loudly
when the library has not been built, and every call raises when the GPU
reports an error.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "liblcbinint_b200.so"

LCBI_OK = 0
LCBI_INVALID_ARGUMENT = 1
LCBI_NUMERICAL_ERROR = 2
LCBI_UNSUPPORTED = 3
LCBI_GPU_ERROR = 16
DEVICE_POINTERS = 1

# The reference's C ABI structs (include/lcbinint/lcbinint.h:46-116) as numpy
# record types with C alignment, for arrays of parameter sets and results.
_PARAMS_HEAD = ("t0", "tE", "umin", "q", "sep", "theta", "rho", "omega", "piEN", "piEE", "piEN_xa", "piEE_xa",
                "ra_xa", "dec_xa", "period_xa", "ecc_xa", "peri_xa", "v_sep", "q2", "sep2", "ang", "ra", "dec",
                "earth_axis", "tfix", "obs_lat", "obs_lon", "limb_darkening_c", "limb_darkening_d")
_PARAMS_TAIL = ("g1", "g2", "g3", "lom_szs", "lom_ar", "xi_1", "xi_2", "omega_xa", "inc_xa", "phi_xa")
PARAMS_DTYPE = np.dtype([(n, "f8") for n in _PARAMS_HEAD] + [("orbital_motion_mode", "i4")] +
                        [(n, "f8") for n in _PARAMS_TAIL], align=True)
OPTIONS_DTYPE = np.dtype([("parallax_mode", "i4"), ("orbit_pair", "i4"), ("center_of_mass", "i4"),
                          ("caustic_bins", "i4"), ("source_bins", "i4"), ("mode", "i4"), ("vbm_compatible", "i4"),
                          ("xallarap_param_type", "i4"), ("grid_ratio", "f8"), ("polar_source_bins", "i4"),
                          ("polar_grid_ratio", "f8"), ("point_source_threshold", "f8"),
                          ("hexadecapole_threshold", "f8"), ("adaptive_hex_threshold", "f8"),
                          ("adaptive_source_bins", "i4"), ("max_source_bins", "i4"), ("finite_source_tol", "f8"),
                          ("finite_source_reltol", "f8")], align=True)
RESULT_DTYPE = np.dtype([("magnification", "f8"), ("point_source_magnification", "f8"),
                         ("finite_source_magnification", "f8"), ("source_x", "f8"), ("source_y", "f8"),
                         ("image_count", "i4"), ("finite_source_error_estimate", "f8"),
                         ("finite_source_refinement_level", "i4"), ("finite_source_converged", "i4")], align=True)
ARRAYS_KEYWORD_ROUTE = 1


def default_params(n: int = 1) -> np.ndarray:
    """lcbi_default_params (lcbinint.h:118) for n parameter sets."""
    p = np.zeros(n, dtype=PARAMS_DTYPE)
    p["tE"] = 1.0
    p["q"] = 1.0
    p["sep"] = 1.0
    p["lom_ar"] = 1.0
    return p


def default_options() -> np.ndarray:
    """lcbi_default_options (lcbinint.h:119), as a one-element array."""
    o = np.zeros(1, dtype=OPTIONS_DTYPE)
    o["orbit_pair"] = 23
    o["caustic_bins"] = 1400
    o["source_bins"] = 50
    o["mode"] = 4
    o["grid_ratio"] = 4.0
    o["point_source_threshold"] = 20.0
    o["hexadecapole_threshold"] = 3.0
    o["adaptive_hex_threshold"] = 0.001
    o["max_source_bins"] = 400
    return o


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_vp = C.c_void_p

_lock = threading.Lock()
_lib = None


class LibraryMissing(RuntimeError):
    pass


def lib() -> C.CDLL:
    """The loaded CUDA library (built by `python -m lcbinint_b200.build`)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not LIB_PATH.exists():
                    raise LibraryMissing(
                        f"{LIB_PATH} is missing: build it with `python -m lcbinint_b200.build`")
                L = C.CDLL(str(LIB_PATH))
                _declare(L)
                _lib = L
    return _lib


def _declare(L):
    L.lcbi_gpu_create.argtypes = [C.c_int, C.POINTER(_vp)]
    L.lcbi_gpu_create.restype = C.c_int
    L.lcbi_gpu_destroy.argtypes = [_vp]
    L.lcbi_gpu_destroy.restype = None
    L.lcbi_gpu_last_error.argtypes = [_vp]
    L.lcbi_gpu_last_error.restype = C.c_char_p
    L.lcbi_gpu_launch_count.argtypes = [_vp]
    L.lcbi_gpu_launch_count.restype = C.c_int64
    L.lcbi_gpu_binary_mag0.argtypes = [_vp, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_uint]
    L.lcbi_gpu_binary_mag0.restype = C.c_int
    L.lcbi_gpu_binary_mag0_derivatives.argtypes = [_vp, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                                   C.c_uint]
    L.lcbi_gpu_binary_mag0_derivatives.restype = C.c_int
    L.lcbi_gpu_binary_mag.argtypes = [_vp, _vp, C.c_int32, _vp, C.c_int32, C.c_int64, _vp, _vp, C.c_uint]
    L.lcbi_gpu_binary_mag.restype = C.c_int
    L.lcbi_gpu_binary_inverse_ray.argtypes = [_vp, _vp, C.c_int64] + [_vp] * 8
    L.lcbi_gpu_binary_inverse_ray.restype = C.c_int
    L.lcbi_gpu_light_curves.argtypes = [_vp, _vp, C.c_int32, _vp, _vp, _vp, _vp, C.c_int64, _vp, _vp, _vp]
    L.lcbi_gpu_light_curves.restype = C.c_int
    L.lcbi_gpu_set_stream.argtypes = [_vp, _vp]
    L.lcbi_gpu_set_stream.restype = C.c_int
    L.lcbi_gpu_set_timing.argtypes = [_vp, C.c_int]
    L.lcbi_gpu_set_timing.restype = C.c_int
    L.lcbi_gpu_stage_times.argtypes = [_vp, _vp, _vp, C.c_int32]
    L.lcbi_gpu_stage_times.restype = C.c_int
    L.lcbi_gpu_measure_fp64_peak.argtypes = [_vp, _vp]
    L.lcbi_gpu_measure_fp64_peak.restype = C.c_int
    L.lcbi_gpu_set_item_cycles.argtypes = [_vp, C.c_int]
    L.lcbi_gpu_set_item_cycles.restype = C.c_int
    L.lcbi_gpu_set_cell_budget.argtypes = [_vp, C.c_int64]
    L.lcbi_gpu_set_cell_budget.restype = C.c_int
    L.lcbi_gpu_set_seed_block_after.argtypes = [_vp, C.c_int32]
    L.lcbi_gpu_set_seed_block_after.restype = C.c_int
    L.lcbi_gpu_set_ray_precision.argtypes = [_vp, C.c_int32]
    L.lcbi_gpu_set_ray_precision.restype = C.c_int
    L.lcbi_gpu_set_grad_resolution.argtypes = [_vp, C.c_int32]
    L.lcbi_gpu_set_grad_resolution.restype = C.c_int
    L.lcbi_gpu_set_stream_marks.argtypes = [_vp, C.c_int]
    L.lcbi_gpu_set_stream_marks.restype = C.c_int
    L.lcbi_gpu_stream_marks.argtypes = [_vp, _vp, C.c_int32]
    L.lcbi_gpu_stream_marks.restype = C.c_int
    L.lcbi_gpu_set_early_helpers.argtypes = [_vp, C.c_int]
    L.lcbi_gpu_set_early_helpers.restype = C.c_int
    L.lcbi_gpu_set_polar_tiles.argtypes = [_vp, C.c_int]
    L.lcbi_gpu_set_polar_tiles.restype = C.c_int
    L.lcbi_gpu_set_workspace.argtypes = [_vp, C.c_int32, C.c_int32, C.c_int64]
    L.lcbi_gpu_set_workspace.restype = C.c_int
    L.lcbi_gpu_binary_mag_grad.argtypes = [_vp, _vp, C.c_int32, _vp, C.c_int32, C.c_int64, _vp, _vp, _vp, C.c_uint]
    L.lcbi_gpu_binary_mag_grad.restype = C.c_int
    L.lcbi_gpu_light_curves_grad.argtypes = [_vp, _vp, C.c_int32, _vp, _vp, _vp, _vp, C.c_int64, _vp, _vp, _vp, _vp]
    L.lcbi_gpu_light_curves_grad.restype = C.c_int
    L.lcbi_gpu_last_item_cycles.argtypes = [_vp, C.c_int64, _vp]
    L.lcbi_gpu_last_item_cycles.restype = C.c_int
    L.lcbi_gpu_last_ray_counts.argtypes = [_vp, C.c_int64, _vp]
    L.lcbi_gpu_last_ray_counts.restype = C.c_int
    L.lcbi_gpu_binary_mag_noalloc.argtypes = [_vp, _vp, C.c_double, C.c_double, C.c_int64, _vp, _vp, _vp, _vp]
    L.lcbi_gpu_binary_mag_noalloc.restype = C.c_int
    L.lcbi_gpu_magnification_arrays.argtypes = [_vp, C.c_int32, _vp, _vp, _vp, _vp, _vp, C.c_int64, C.c_uint, _vp,
                                                 _vp]
    L.lcbi_gpu_magnification_arrays.restype = C.c_int
    L.lcbi_gpu_autotune.argtypes = [_vp, _vp, C.c_int32, _vp, C.c_int32, C.c_int64, _vp, _vp, C.c_uint, _vp, _vp]
    L.lcbi_gpu_autotune.restype = C.c_int
    L.lcbi_set_earth_ephemeris.argtypes = [C.c_char_p]
    L.lcbi_set_earth_ephemeris.restype = C.c_int
    L.lcbi_gpu_binary_geometry.argtypes = [_vp, C.c_double, C.c_double, C.c_int32, C.c_int32, _vp, _vp]
    L.lcbi_gpu_binary_geometry.restype = C.c_int
    L.lcbi_circular_orbital_motion.argtypes = [C.c_double] * 7 + [_vp]
    L.lcbi_circular_orbital_motion.restype = C.c_int
    L.lcbi_kepler_orbital_motion.argtypes = [C.c_double] * 9 + [_vp]
    L.lcbi_kepler_orbital_motion.restype = C.c_int
    L.lcbi_gpu_binary_image_candidates.argtypes = [_vp, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, C.c_uint]
    L.lcbi_gpu_binary_image_candidates.restype = C.c_int
    L.lcbi_gpu_last_refinement_levels.argtypes = [_vp, C.c_int64, _vp]
    L.lcbi_gpu_last_refinement_levels.restype = C.c_int
    L.lcbi_gpu_workspace_bytes.argtypes = [_vp]
    L.lcbi_gpu_workspace_bytes.restype = C.c_int64
    L.lcbi_gpu_kernel_binary_version.argtypes = [_vp]
    L.lcbi_gpu_kernel_binary_version.restype = C.c_int
    L.lcbi_gpu_set_wait_limit.argtypes = [_vp, C.c_uint32]
    L.lcbi_gpu_set_wait_limit.restype = C.c_int
    L.lcbi_gpu_last_wait_timeouts.argtypes = [_vp, _vp]
    L.lcbi_gpu_last_wait_timeouts.restype = C.c_int
    L.lcbi_gpu_light_curves_grad_device.argtypes = [_vp, _vp, C.c_int32, _vp, _vp, _vp, _vp, C.c_int64, _vp, _vp,
                                                    _vp, _vp]
    L.lcbi_gpu_light_curves_grad_device.restype = C.c_int
    L.lcbi_source_trajectory.argtypes = [_vp, _vp, _vp, C.c_int64, _vp, _vp]
    L.lcbi_source_trajectory.restype = C.c_int


def exported_symbols() -> list[str]:
    """Names of the lcbi_* functions the library exports (checked against include/*.h)."""
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True)
    return sorted({ln.split()[-1] for ln in out.stdout.splitlines() if " T lcbi_" in ln})


class GpuError(RuntimeError):
    pass


class Context:
    """One device context (stream + workspaces).  Not shared across threads."""

    def __init__(self, device: int = 0):
        self._L = lib()
        h = _vp()
        rc = self._L.lcbi_gpu_create(int(device), C.byref(h))
        if rc != LCBI_OK:
            raise GpuError(f"lcbi_gpu_create(device={device}) failed with status {rc}")
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self._L.lcbi_gpu_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int, what: str):
        if rc != LCBI_OK:
            msg = self._L.lcbi_gpu_last_error(self.handle).decode()
            raise GpuError(f"{what} failed (status {rc}): {msg}")

    @property
    def launches(self) -> int:
        return int(self._L.lcbi_gpu_launch_count(self.handle))


_ctx = {}


def context(device: int = 0) -> Context:
    """Per-thread default context for `device`."""
    key = (threading.get_ident(), device)
    c = _ctx.get(key)
    if c is None:
        c = Context(device)
        _ctx[key] = c
    return c


def as_f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64).ravel()
    if n is not None and a.size == 1 and n != 1:
        a = np.full(n, a[0])
    return a


def ptr(a) -> int:
    return a.ctypes.data
