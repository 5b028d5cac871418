"""lcbinint_b200: B200-native drop-in for lcbinint's magnification hot path.

The Python surface mirrors the reference's pybind11 module
(python/lcbinint_pybind.cpp): the same callables, argument names, defaults and
error behaviour.  Every call goes through the C ABI of the in-tree CUDA
library (include/lcbinint_b200.h); nothing is computed on the CPU.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import GpuError, LibraryMissing, context
from .api import (CIRCULAR, KEPLER, STATIC, EventCoordinates, GeometryBranches, GeometryCurve, LightCurve,
                  LightCurveFunc,
                  LightCurveInfo, LimbDarkening, Options, binary_geometry, binary_inverse_ray,
                  binary_inverse_ray_batch, binary_mag, circular_orbital_motion, kepler_orbital_motion, light_curves,
                  magnification_arrays, set_earth_ephemeris)

__all__ = [
    "binary_mag0",
    "binary_mag0_batch",
    "binary_inverse_ray",
    "binary_inverse_ray_batch",
    "binary_mag",
    "light_curves",
    "magnification_arrays",
    "binary_geometry",
    "GeometryBranches",
    "GeometryCurve",
    "circular_orbital_motion",
    "kepler_orbital_motion",
    "set_earth_ephemeris",
    "LightCurve",
    "LightCurveFunc",
    "LightCurveInfo",
    "LimbDarkening",
    "Options",
    "EventCoordinates",
    "STATIC",
    "CIRCULAR",
    "KEPLER",
    "GpuError",
    "LibraryMissing",
    "context",
]


def binary_mag0_batch(separation, mass_ratio, y1, y2, *, device: int = 0, return_images: bool = False):
    """Point-source magnification of many source positions in one launch.

    Arrays broadcast against each other.  Same convention as `binary_mag0`.
    """
    s, q, a, b = np.broadcast_arrays(separation, mass_ratio, y1, y2)
    shape = s.shape
    s, q, a, b = (_lib.as_f64(v) for v in (s, q, a, b))
    n = s.size
    A = np.empty(n)
    nimg = np.empty(n, dtype=np.int32)
    status = np.empty(n, dtype=np.int32)
    ctx = context(device)
    rc = ctx._L.lcbi_gpu_binary_mag0(ctx.handle, n, _lib.ptr(s), _lib.ptr(q), _lib.ptr(a), _lib.ptr(b),
                                     _lib.ptr(A), _lib.ptr(nimg), _lib.ptr(status), 0)
    ctx.check(rc, "lcbi_gpu_binary_mag0")
    if return_images:
        return A.reshape(shape), nimg.reshape(shape)
    return A.reshape(shape)


def binary_mag0(separation: float, mass_ratio: float, y1: float, y2: float) -> float:
    """Binary point-source magnification in VBMicrolensing BinaryMag0 coordinates.

    Mirrors lcbinint.binary_mag0 (python/lcbinint_pybind.cpp:3819-3824):
    mass_ratio < 1 puts the heavier lens at -separation; mass_ratio > 1 is
    inverted; (y1, y2) is the source in the centre-of-mass frame.
    """
    return float(binary_mag0_batch(separation, mass_ratio, y1, y2).reshape(-1)[0])
