"""PyTorch wrapper: the mirror of the reference's ``fastprox.torch.tv_iso`` /
``tv_aniso`` (bindings/python/fastprox/torch.py:305-351, 363-524) on the
B200 kernels, through the C ABI on the tensor's data pointers and current
CUDA stream.

``tv_iso(x, gamma, ndim=2, weights=None, pixel_weights=None, tol=1e-6,
max_iter=1000, return_info=False)`` solves the isotropic TV prox of every image
of the last ``ndim`` axes of ``x`` and is differentiable in ``x`` and
``gamma`` (a number or a tensor broadcasting to the batch shape): the
backward pass is the implicit-differentiation VJP on the device (``fp_vjp``),
one linear solve on the solution's flat regions, with memory independent of
the iteration count. ``tv_aniso`` solves anisotropic TV, differentiable the
same way (its VJP averages over the solution's constant components).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi
from .image_tv import IterInfo, TVAniso, TVIso


def _gamma_per_image(gamma, x, ndim):
    batch = tuple(x.shape[:-ndim])
    g = gamma if isinstance(gamma, torch.Tensor) else torch.as_tensor(np.asarray(gamma, np.float64))
    g = g.to(dtype=x.dtype, device=x.device)
    if g.numel() == 1:
        return g.reshape(()), True
    if torch.broadcast_shapes(g.shape, batch) != batch:
        raise ValueError(f"gamma must be a number or broadcast to the batch shape {batch}")
    return g.expand(batch).contiguous(), False


class _DeviceTV(torch.autograd.Function):
    """forward: fp_prox (or fp_prox_steps) with keep_structure; backward:
    fp_vjp at the kept point (the reference's _DeviceTV, torch.py:466-524)."""

    @staticmethod
    def forward(ctx, op, cfg, x, gamma):
        scalar = gamma.dim() == 0
        xc = x.detach().contiguous()
        z = torch.empty_like(xc)
        ws = op.workspace(xc, keep=True)
        L = capi.lib()
        stream = torch.cuda.current_stream(x.device).cuda_stream if x.is_cuda else None
        if x.is_cuda:
            capi.check(L.fp_workspace_set_stream(ws, C.c_void_p(stream)), "set_stream")
        opt = capi.options(tol=cfg["tol"], max_iter=cfg["max_iter"], keep=True)
        xr, zr = capi.ArrayRef(xc), capi.ArrayRef(z)
        if scalar:
            st = L.fp_prox(op._op, float(gamma), xr.ref(), zr.ref(), C.byref(opt), ws, None)
        else:
            st = L.fp_prox_steps(op._op, capi.ArrayRef(gamma.detach().contiguous()).ref(), xr.ref(), zr.ref(),
                                 C.byref(opt), ws)
        capi.check(st, "fp_prox", (capi.FP_OK, capi.FP_ENOTCONV))
        B = int(np.prod(x.shape[:x.dim() - op.k])) if x.dim() > op.k else 1
        gaps, its, zerr = np.zeros(B), np.zeros(B, np.int32), np.zeros(B)
        capi.check(L.fp_workspace_image_info(ws, gaps.ctypes.data_as(C.POINTER(C.c_double)),
                                             its.ctypes.data_as(C.POINTER(C.c_int)),
                                             zerr.ctypes.data_as(C.POINTER(C.c_double)), B), "image_info")
        cfg["info"] = IterInfo(float(np.nansum(gaps)), int(its.max(initial=0)), st == capi.FP_OK, gaps, its, zerr)
        ctx.op, ctx.ws, ctx.scalar = op, ws, scalar
        ctx.gshape = gamma.shape
        return z

    @staticmethod
    def backward(ctx, gz):
        L = capi.lib()
        g = gz.detach().contiguous()
        gx = torch.empty_like(g)
        gg = C.c_double(0.0)
        if g.is_cuda:
            capi.check(L.fp_workspace_set_stream(ctx.ws, C.c_void_p(torch.cuda.current_stream(g.device).cuda_stream)),
                       "set_stream")
        capi.check(L.fp_vjp(ctx.op._op, ctx.ws, capi.ArrayRef(g).ref(), capi.ArrayRef(gx).ref(), C.byref(gg), None),
                   "fp_vjp")
        ggamma = None
        if ctx.needs_input_grad[3]:
            if not ctx.scalar:
                raise NotImplementedError("the gradient of one step per image is summed by fp_vjp; pass one gamma")
            ggamma = torch.as_tensor(gg.value, dtype=g.dtype, device=g.device).reshape(ctx.gshape)
        return None, None, gx, ggamma


def tv_iso(x, gamma=1.0, *, ndim=2, weights=None, pixel_weights=None, tol=1e-6, max_iter=1000, return_info=False):
    """Isotropic TV prox of the last ``ndim`` axes of ``x`` (differentiable in
    ``x`` and a scalar ``gamma``)."""
    if not isinstance(x, torch.Tensor):
        raise TypeError("x must be a torch.Tensor")
    if ndim not in (2, 3) or x.dim() < ndim:
        raise ValueError("ndim must be 2 or 3 and x must have at least ndim dimensions")
    op = TVIso(ndim, weights, None if pixel_weights is None else np.asarray(
        pixel_weights.detach().cpu() if isinstance(pixel_weights, torch.Tensor) else pixel_weights, np.float64))
    g, _ = _gamma_per_image(gamma, x, ndim)
    cfg = {"tol": float(tol), "max_iter": int(max_iter)}
    z = _DeviceTV.apply(op, cfg, x, g)
    return (z, cfg["info"]) if return_info else z


def tv_aniso(x, gamma=1.0, *, ndim=2, weights=None, edge_weights=None, tol=1e-6, max_iter=1000, return_info=False):
    """Anisotropic TV prox of the last ``ndim`` axes of ``x`` (differentiable
    in ``x`` and a scalar ``gamma``: the backward pass averages the cotangent
    over the solution's constant components, tv_aniso.cpp:1398-1440)."""
    if not isinstance(x, torch.Tensor):
        raise TypeError("x must be a torch.Tensor")
    if ndim not in (2, 3) or x.dim() < ndim:
        raise ValueError("ndim must be 2 or 3 and x must have at least ndim dimensions")
    op = TVAniso(ndim, weights, None if edge_weights is None else np.asarray(
        edge_weights.detach().cpu() if isinstance(edge_weights, torch.Tensor) else edge_weights, np.float64))
    g, _ = _gamma_per_image(gamma, x, ndim)
    cfg = {"tol": float(tol), "max_iter": int(max_iter)}
    z = _DeviceTV.apply(op, cfg, x, g)
    return (z, cfg["info"]) if return_info else z
