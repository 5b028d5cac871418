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
