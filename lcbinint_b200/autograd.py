"""Gradients of binary-lens light curves for torch: a torch.autograd.Function
over the library's adjoint entry point (lcbi_gpu_light_curves_grad).

    A = light_curve_magnification(params, times)        # params: (M, 8) float64
    A.sum().backward()                                   # params.grad: dA/dparams

params[m] = (t0, tE, u0, alpha, s, q, rho, Gamma) in the VBM convention of
lcbinint.LightCurve (python/lcbinint_pybind.cpp:1140-1157) with linear limb
darkening Gamma; times is (M, K) or (K,) (shared).  The forward is the
library's batched light-curve pass; its backward uses the per-epoch gradients
the same call computed, so one call gives magnifications and gradients.
No reference counterpart: the reference differences its forward.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .api import LimbDarkening, Options


def light_curves_with_grad(params, times, options: Options = None, *, device: int = 0, with_grad: bool = True):
    """Host-array form: params (M, 8), times (M, K) -> (A (M, K), dA (M, K, 8) or None, method, status)."""
    P = np.ascontiguousarray(params, dtype=np.float64).reshape(-1, 8)
    M = P.shape[0]
    T = np.asarray(times, dtype=np.float64)
    if T.ndim == 1:
        T = np.broadcast_to(T, (M, T.size))
    T = np.ascontiguousarray(T)
    K = T.shape[1]
    n = M * K
    first = np.arange(M, dtype=np.int64) * K
    count = np.full(M, K, dtype=np.int32)
    A = np.empty(n)
    dA = np.empty((n, 8)) if with_grad else None
    method = np.empty(n, dtype=np.int32)
    status = np.empty(n, dtype=np.int32)
    opt = options or Options()
    st = opt.fs_settings(LimbDarkening())
    ctx = _lib.context(device)
    rc = ctx._L.lcbi_gpu_light_curves_grad(ctx.handle, C.byref(st), M, _lib.ptr(P), _lib.ptr(first),
                                           _lib.ptr(count), _lib.ptr(T), n, _lib.ptr(A),
                                           _lib.ptr(dA) if with_grad else None, _lib.ptr(method), _lib.ptr(status))
    ctx.check(rc, "lcbi_gpu_light_curves_grad")
    return (A.reshape(M, K), dA.reshape(M, K, 8) if with_grad else None, method.reshape(M, K),
            status.reshape(M, K))


def _function():
    import torch

    class LightCurveMagnification(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, times, options):
            dev = params.device.index if (params.is_cuda and params.device.index is not None) else 0
            A, dA, _, _ = light_curves_with_grad(params.detach().cpu().numpy(), times.detach().cpu().numpy(),
                                                 options, device=dev, with_grad=params.requires_grad)
            if dA is not None:
                ctx.save_for_backward(torch.from_numpy(dA).to(params.device))
            return torch.from_numpy(A).to(params.device)

        @staticmethod
        def backward(ctx, grad_A):
            dA, = ctx.saved_tensors
            return (grad_A.unsqueeze(-1) * dA).sum(dim=1), None, None

    return LightCurveMagnification


_FN = None


def light_curve_magnification(params, times, options: Options = None):
    """Differentiable magnifications (M, K) of M static binary light curves."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(params, times, options)
