"""Gradients of binary-lens light curves for torch: a torch.autograd.Function
over the library's adjoint entry point (lcbi_gpu_light_curves_grad).

    A = light_curve_magnification(params, times)        # params: (M, 8) float64
    A.sum().backward()                                   # params.grad: dA/dparams

params[m] = (t0, tE, u0, alpha, s, q, rho, Gamma) in the VBM convention of
lcbinint.LightCurve (python/lcbinint_pybind.cpp:1140-1157) with linear limb
darkening Gamma; times is (M, K) or (K,) (shared).  The forward is the
library's batched light-curve pass; its backward uses the per-epoch gradients
the same call computed, so one call gives magnifications and gradients.  With
times on a CUDA device the per-epoch arrays (times, magnifications, gradients)
never leave it; only the (M, 8) parameters are read on the host.
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


def light_curves_with_grad_device(params, times, options: Options = None, *, with_grad: bool = True):
    """Device-tensor form (lcbi_gpu_light_curves_grad_device): times is a CUDA
    tensor (M, K) or (K,); A (M, K), dA (M, K, 8) or None, method and status
    come back as CUDA tensors on the same device, ordered on torch's current
    stream.  params (M, 8) may live anywhere: its 64 bytes per model are read
    on the host, where the caustic models are planned."""
    import torch
    dev = times.device
    P = np.ascontiguousarray(params.detach().to("cpu", torch.float64).numpy()).reshape(-1, 8)
    M = P.shape[0]
    T = times.detach().to(torch.float64)
    if T.dim() == 1:
        T = T.unsqueeze(0).expand(M, T.shape[0])
    T = T.contiguous()
    K = T.shape[1]
    n = M * K
    first = np.arange(M, dtype=np.int64) * K
    count = np.full(M, K, dtype=np.int32)
    A = torch.empty((M, K), dtype=torch.float64, device=dev)
    dA = torch.empty((M, K, 8), dtype=torch.float64, device=dev) if with_grad else None
    method = torch.empty((M, K), dtype=torch.int32, device=dev)
    status = torch.empty((M, K), dtype=torch.int32, device=dev)
    st = (options or Options()).fs_settings(LimbDarkening())
    ctx = _lib.context(dev.index if dev.index is not None else 0)
    L = ctx._L
    L.lcbi_gpu_set_stream(ctx.handle, torch.cuda.current_stream(dev).cuda_stream)
    try:
        rc = L.lcbi_gpu_light_curves_grad_device(ctx.handle, C.byref(st), M, _lib.ptr(P), _lib.ptr(first),
                                                 _lib.ptr(count), T.data_ptr(), n, A.data_ptr(),
                                                 dA.data_ptr() if with_grad else None, method.data_ptr(),
                                                 status.data_ptr())
    finally:
        L.lcbi_gpu_set_stream(ctx.handle, None)
    ctx.check(rc, "lcbi_gpu_light_curves_grad_device")
    return A, dA, method, status


def _function():
    import torch

    class LightCurveMagnification(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, times, options):
            if times.is_cuda:
                # Per-epoch arrays stay on the device.
                A, dA, _, _ = light_curves_with_grad_device(params, times, options,
                                                            with_grad=params.requires_grad)
                if dA is not None:
                    ctx.save_for_backward(dA.to(params.device))
                return A.to(params.device)
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
