"""PyTorch wrapper: the mirror of the reference's ``fastprox.torch.tv_iso`` /
``tv_aniso`` (bindings/python/fastprox/torch.py:305-524) on the B200 kernels,
through the C ABI on the tensor's data pointers and current CUDA stream.

``tv_iso(x, gamma, *, ndim=2, weights=None, pixel_weights=None, tol=None,
ztol=None, max_iter=1000, warm_start=None, return_info=False, deriv_tol=None,
deriv_max_iter=10000, warn=True)`` solves the isotropic TV prox of every image
of the last ``ndim`` axes of ``x``; ``tv_aniso`` (with ``edge_weights``) the
anisotropic one. Both are differentiable, reverse and forward mode, in ``x``,
``gamma`` (a number or one step per image: a tensor broadcasting to the batch
shape ``x.shape[:-ndim]``), the axis ``weights`` and the pixel or edge weights
(tensors that require grad): the reverse pass is the implicit-differentiation
VJP on the device (``fp_vjp``: one linear solve on the solution's flat regions
for isotropic TV, component averages for anisotropic TV), the forward pass
``fp_jvp``; their memory does not grow with the iteration count.

* ``tol``: each image stops when its duality gap is at most
  tol |x|^2 / 2 (default 1e-6); ``ztol`` asks for that relative error of z
  instead (tol = ztol^2); not both.
* ``pixel_weights`` (isotropic) broadcast to ``x.shape``, ``edge_weights``
  (anisotropic) have shape (ndim, ...) broadcasting to (ndim, *x.shape): one
  map for every image (one operator, one call) or one per image (an operator
  and a call per image).
* ``warm_start``: the ``dual`` of an earlier call, shape (ndim, *x.shape).
* ``deriv_tol`` / ``deriv_max_iter``: the derivatives' linear solves
  (``fp_workspace_set_deriv_tol``); by default each image's solve stops at the
  relative error of z its gap certifies.
* A solve that stops at ``max_iter`` warns (``ConvergenceWarning``) unless
  ``warn=False``.
"""

from __future__ import annotations

import ctypes as C
import math
import warnings

import numpy as np
import torch

from . import capi
from .image_tv import IterInfo, TVAniso, TVIso


class ConvergenceWarning(UserWarning):
    """An image-TV solve stopped at max_iter before its tolerance; the message
    gives the certified relative error of z (the reference's
    fastprox.ConvergenceWarning)."""


def _call_tol(tol, ztol):
    if tol is not None and ztol is not None:
        raise ValueError("pass tol or ztol, not both")
    if ztol is not None:
        z = float(ztol)
        if not z >= 0.0:
            raise ValueError("ztol must be >= 0")
        return z * z
    t = 1e-6 if tol is None else float(tol)
    if not t >= 0.0:
        raise ValueError("tol must be >= 0")
    return t


def _axis_weights(weights, ndim):
    """The axis weights as floats, and the tensor to differentiate, if any."""
    wt = None
    if weights is None:
        w = [1.0] * ndim
    elif isinstance(weights, torch.Tensor) and weights.is_floating_point():
        wt = weights
        w = [float(a) for a in weights.detach().cpu().reshape(-1)]
    else:
        w = [float(a) for a in np.atleast_1d(np.asarray(weights, np.float64))]
    if len(w) == 1:
        w = w * ndim
    if len(w) != ndim or min(w) < 0 or not all(math.isfinite(a) for a in w):
        raise ValueError("weights must be one or ndim finite values >= 0")
    return w, wt


def _per_image(gamma, x, ndim):
    """gamma as one value per image, (B,), in the graph of gamma (the
    reference's _per_image, torch.py:443-463)."""
    batch = tuple(x.shape[:-ndim])
    g = gamma if isinstance(gamma, torch.Tensor) else torch.as_tensor(np.asarray(gamma, np.float64))
    if not g.is_floating_point():
        g = g.to(torch.float64)
    g = g.to(dtype=x.dtype, device=x.device)
    if g.numel() == 1:
        g = g.reshape(())
    try:
        if torch.broadcast_shapes(g.shape, batch) != batch:
            raise RuntimeError
    except RuntimeError:
        raise ValueError(f"gamma must be a number or broadcast to the batch shape {batch}, "
                         f"got shape {tuple(g.shape)}") from None
    gd = g.detach()
    if bool(((gd < 0) | ~torch.isfinite(gd)).any()):
        raise ValueError("gamma must be finite and >= 0")
    return g.expand(batch).reshape(-1)


def _spatial(sw, x, ndim, iso):
    """Pixel weights broadcasting to x.shape, or edge weights of shape
    (ndim, ...) broadcasting to (ndim, *x.shape) (the reference's _spatial,
    torch.py:416-441), in the graph of sw: one map for the batch, shape
    (*img) or (ndim, *img), when sw has no batch extent, else one per image,
    (B, *img) or (ndim, B, *img)."""
    name = "pixel_weights" if iso else "edge_weights"
    full = tuple(x.shape) if iso else (ndim, *x.shape)
    t = sw if isinstance(sw, torch.Tensor) else torch.as_tensor(np.asarray(sw, np.float64))
    t = t.to(dtype=x.dtype, device=x.device)
    try:
        if not iso:  # the leading axis is the image axis; the rest broadcasts to x
            if t.dim() < 1 or t.shape[0] != ndim or t.dim() - 1 > x.dim():
                raise RuntimeError
            t = t.reshape((ndim,) + (1,) * (x.dim() + 1 - t.dim()) + tuple(t.shape[1:]))
        if torch.broadcast_shapes(t.shape, full) != full:
            raise RuntimeError
    except RuntimeError:
        what = "broadcast to" if iso else f"have shape ({ndim}, ...) broadcasting to"
        raise ValueError(f"{name} must {what} {full}, got shape {tuple(sw.shape) if hasattr(sw, 'shape') else ()}") \
            from None
    td = t.detach()
    if bool(((td < 0) | ~torch.isfinite(td)).any()):
        raise ValueError(f"{name} must be finite and >= 0")
    img = tuple(x.shape[-ndim:])
    lead = 0 if iso else 1
    t = t.reshape(tuple(t.shape[:lead]) + (1,) * (len(full) - t.dim()) + tuple(t.shape[lead:]))
    nb = x.dim() - ndim
    if all(e == 1 for e in t.shape[lead:lead + nb]):  # one map for the batch
        one = t.reshape(tuple(t.shape[:lead]) + tuple(t.shape[lead + nb:]))
        return one.expand(((ndim,) if not iso else ()) + img), True
    return t.expand(full).reshape((-1,) + img if iso else (ndim, -1) + img), False


class _Solve:
    """One operator's solve of a group of images (all of them, or one image
    with its own weight map), keeping its workspace for the derivatives."""

    def __init__(self, iso, k, w, spatial_np, xg, gam, cfg, dual):
        Op = TVIso if iso else TVAniso
        self.op = Op(k, w, spatial_np)
        self.k = k
        L = capi.lib()
        self.ws = self.op.workspace(xg, keep=True)
        self._stream(xg)
        capi.check(L.fp_workspace_set_warm(self.ws, 0), "set_warm")
        if dual is not None:
            capi.check(L.fp_workspace_set_dual(self.ws, capi.ArrayRef(dual.contiguous()).ref()), "set_dual")
        if cfg.deriv_tol is not None:
            capi.check(L.fp_workspace_set_deriv_tol(self.ws, cfg.deriv_tol, cfg.deriv_max_iter), "deriv_tol")
        self.z = torch.empty_like(xg)
        opt = capi.options(tol=cfg.tol, max_iter=cfg.max_iter, keep=True)
        st = L.fp_prox_steps(self.op._op, capi.ArrayRef(gam.contiguous()).ref(), capi.ArrayRef(xg).ref(),
                             capi.ArrayRef(self.z).ref(), C.byref(opt), self.ws)
        capi.check(st, "fp_prox_steps", (capi.FP_OK, capi.FP_ENOTCONV))
        B = xg.shape[0]
        self.gaps, self.iters, self.zerr = np.zeros(B), np.zeros(B, np.int32), np.zeros(B)
        capi.check(L.fp_workspace_image_info(self.ws, self.gaps.ctypes.data_as(C.POINTER(C.c_double)),
                                             self.iters.ctypes.data_as(C.POINTER(C.c_int)),
                                             self.zerr.ctypes.data_as(C.POINTER(C.c_double)), B), "image_info")
        self.dual = torch.empty((k,) + tuple(xg.shape), dtype=xg.dtype, device=xg.device)
        capi.check(L.fp_workspace_get_dual(self.ws, capi.ArrayRef(self.dual).ref()), "get_dual")
        self.converged = st == capi.FP_OK

    def _stream(self, t):
        if t.is_cuda:
            with torch.cuda.device(t.device):
                s = torch.cuda.current_stream().cuda_stream
            capi.check(capi.lib().fp_workspace_set_stream(self.ws, C.c_void_p(s)), "set_stream")

    def vjp(self, g):
        """(gx, per-image step gradients (B,), per-image axis-weight gradients
        (B, k), the weight map's gradient (nparams - k,))."""
        L = capi.lib()
        self._stream(g)
        g = g.contiguous()
        gx = torch.empty_like(g)
        P = self.op.nparams
        gp = np.zeros(P)
        capi.check(L.fp_vjp(self.op._op, self.ws, capi.ArrayRef(g).ref(), capi.ArrayRef(gx).ref(), None,
                            capi.ArrayRef(gp).ref()), "fp_vjp")
        B = g.shape[0]
        gg, gw = np.zeros(B), np.zeros((B, self.k))
        capi.check(L.fp_b200_vjp_images(self.ws, gg.ctypes.data_as(C.POINTER(C.c_double)),
                                        gw.ctypes.data_as(C.POINTER(C.c_double)), B), "vjp_images")
        return gx, gg, gw, gp[self.k:]

    def jvp(self, dx, dgamma, dparams):
        """dz for the tangent (dx or None, one dgamma for every image, the
        parameters' tangent or None)."""
        L = capi.lib()
        self._stream(self.z)
        out = torch.empty_like(self.z)
        dxr = None if dx is None else capi.ArrayRef(dx.contiguous())
        dpr = None if dparams is None else capi.ArrayRef(np.ascontiguousarray(dparams, np.float64))
        capi.check(L.fp_jvp(self.op._op, self.ws, None if dxr is None else dxr.ref(), float(dgamma),
                            None if dpr is None else dpr.ref(), capi.ArrayRef(out).ref()), "fp_jvp")
        return out


class _Cfg:
    def __init__(self, iso, k, w, tol, max_iter, deriv_tol, deriv_max_iter, uniform):
        self.iso, self.k, self.w = iso, k, w
        self.tol, self.max_iter = float(tol), int(max_iter)
        self.deriv_tol = None if deriv_tol is None else float(deriv_tol)
        self.deriv_max_iter = int(deriv_max_iter)
        self.uniform = uniform
        self.info = None


class _DeviceTV(torch.autograd.Function):
    """forward: fp_prox_steps with keep_structure (one call, or one per image
    when every image has its own weight map); backward: fp_vjp, forward mode:
    fp_jvp at the kept point (the reference's _DeviceTV, torch.py:466-524)."""

    @staticmethod
    def forward(ctx, cfg, x, gamma, wt, sw, warm):
        k = cfg.k
        img = tuple(x.shape[-k:])
        xb = x.detach().reshape((-1,) + img).contiguous()
        gam = gamma.detach().to(torch.float64)
        B = xb.shape[0]
        dual = None if warm is None else warm.reshape((k, B) + img)
        swd = None if sw is None else sw.detach()
        solves = []
        if sw is None or cfg.uniform:
            sp = None if swd is None else swd.cpu().double().numpy()
            solves.append((slice(0, B), _Solve(cfg.iso, k, cfg.w, sp, xb, gam, cfg, dual)))
        else:  # one operator per image: its own weight map
            for b in range(B):
                sp = (swd[b] if cfg.iso else swd[:, b]).cpu().double().numpy()
                d = None if dual is None else dual[:, b:b + 1]
                solves.append((slice(b, b + 1), _Solve(cfg.iso, k, cfg.w, sp, xb[b:b + 1], gam[b:b + 1], cfg, d)))
        z = torch.cat([s.z for _, s in solves]) if len(solves) > 1 else solves[0][1].z
        gaps = np.concatenate([s.gaps for _, s in solves])
        iters = np.concatenate([s.iters for _, s in solves])
        zerr = np.concatenate([s.zerr for _, s in solves])
        dl = torch.cat([s.dual for _, s in solves], dim=1) if len(solves) > 1 else solves[0][1].dual
        cfg.info = IterInfo(float(np.nansum(gaps)) if not np.isnan(gaps).all() else float("nan"),
                            int(iters.max(initial=0)), all(s.converged for _, s in solves), gaps, iters, zerr,
                            dl.reshape((k,) + tuple(x.shape)))
        ctx.cfg, ctx.solves, ctx.shape, ctx.img = cfg, solves, tuple(x.shape), img
        ctx.wt_shape = None if wt is None else tuple(wt.shape)
        ctx.sw_shape = None if sw is None else tuple(sw.shape)
        return z.reshape(x.shape)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, c):
        cfg = ctx.cfg
        cb = c.reshape((-1,) + ctx.img)
        B = cb.shape[0]
        gx = torch.empty_like(cb)
        gg = np.zeros(B)
        gw = np.zeros(cfg.k)
        gmaps = []
        for sl, s in ctx.solves:
            gxi, ggi, gwi, gmi = s.vjp(cb[sl])
            gx[sl] = gxi
            gg[sl] = ggi
            gw += gwi.sum(axis=0)
            gmaps.append(gmi)
        out_x = gx.reshape(ctx.shape) if ctx.needs_input_grad[1] else None
        out_g = torch.as_tensor(gg, dtype=c.dtype, device=c.device) if ctx.needs_input_grad[2] else None
        out_w = None
        if ctx.wt_shape is not None and ctx.needs_input_grad[3]:
            v = torch.as_tensor(gw, dtype=c.dtype, device=c.device)
            n = int(np.prod(ctx.wt_shape, dtype=np.int64))
            out_w = v.sum().reshape(ctx.wt_shape) if n == 1 else v.reshape(ctx.wt_shape)
        out_s = None
        if ctx.sw_shape is not None and ctx.needs_input_grad[4]:
            k, img = cfg.k, ctx.img
            if cfg.uniform:
                out_s = torch.as_tensor(gmaps[0], dtype=c.dtype, device=c.device).reshape(ctx.sw_shape)
            elif cfg.iso:
                out_s = torch.stack([torch.as_tensor(m, dtype=c.dtype, device=c.device).reshape(img)
                                     for m in gmaps])
            else:
                out_s = torch.stack([torch.as_tensor(m, dtype=c.dtype, device=c.device).reshape((k,) + img)
                                     for m in gmaps], dim=1)
        return None, out_x, out_g, out_w, out_s, None

    @staticmethod
    def jvp(ctx, _cfg, dx, dgamma, dwt, dsw, _dwarm):
        cfg = ctx.cfg
        k, img = cfg.k, ctx.img
        dxb = None if dx is None else dx.reshape((-1,) + img)
        dw = None
        if dwt is not None:
            vals = [float(a) for a in dwt.detach().cpu().reshape(-1)]
            dw = vals * k if len(vals) == 1 else vals
        outs = []
        for sl, s in ctx.solves:
            dp = None
            if dw is not None or dsw is not None:
                tail = s.op.nparams - k
                mp = np.zeros(tail)
                if dsw is not None:
                    if cfg.uniform:
                        mp = dsw.detach().cpu().double().numpy().reshape(-1)
                    else:
                        b = sl.start
                        m = dsw[b] if cfg.iso else dsw[:, b]
                        mp = m.detach().cpu().double().numpy().reshape(-1)
                dp = np.concatenate([np.asarray(dw if dw is not None else [0.0] * k, np.float64), mp])
            dz = s.jvp(None if dxb is None else dxb[sl], 0.0, dp)
            if dgamma is not None:
                # dz/dgamma_b per image (fp_jvp takes one dgamma): the derivative
                # at dgamma = 1 for every image, scaled by each image's tangent
                dzg = s.jvp(None, 1.0, None)
                gb = dgamma.detach().reshape(-1)[sl].to(dzg.dtype)
                dz = dz + dzg * gb.reshape((-1,) + (1,) * k)
            outs.append(dz)
        return (torch.cat(outs) if len(outs) > 1 else outs[0]).reshape(ctx.shape)


def _device_tv(iso, x, gamma, ndim, weights, spatial, tol, ztol, max_iter, warm_start, return_info, deriv_tol,
               deriv_max_iter, warn, who):
    if not isinstance(x, torch.Tensor):
        raise TypeError("x must be a torch.Tensor")
    if x.dtype not in (torch.float32, torch.float64):
        raise TypeError("x must be float32 or float64")
    if ndim not in (2, 3):
        raise ValueError("ndim must be 2 or 3")
    if x.dim() < ndim:
        raise ValueError(f"needs a tensor with at least {ndim} dimensions")
    t = _call_tol(tol, ztol)
    if max_iter < 0:
        raise ValueError("max_iter must be >= 0")
    w, wt = _axis_weights(weights, ndim)
    gb = _per_image(gamma, x, ndim)
    warm = None
    if warm_start is not None:
        warm = torch.as_tensor(warm_start).to(dtype=x.dtype, device=x.device)
        if tuple(warm.shape) != (ndim, *x.shape):
            raise ValueError(f"warm_start must have shape {(ndim, *x.shape)}")
    if deriv_tol is not None and not deriv_tol > 0:
        raise ValueError("deriv_tol must be > 0 or None")
    sw, uniform = (None, True) if spatial is None else _spatial(spatial, x, ndim, iso)
    cfg = _Cfg(iso, ndim, w, t, max(int(max_iter), 1), deriv_tol, deriv_max_iter, uniform)
    if x.numel() == 0:  # an empty batch: an empty result, in the graph of every input
        z = x.clone()
        for p in (gb, wt, sw):
            if p is not None:
                z = z + 0 * p.sum()
        info = IterInfo(0.0, 0, True, np.zeros(0), np.zeros(0, np.int32), np.zeros(0),
                        torch.zeros((ndim, *x.shape), dtype=x.dtype, device=x.device))
        return (z, info) if return_info else z
    if bool(torch.isinf(x.detach()).any()):
        raise ValueError("x contains ±Inf; image operators reject infinite values")
    z = _DeviceTV.apply(cfg, x, gb, wt, sw, warm)
    info = cfg.info
    if warn and not info.converged:
        worst = float(np.nanmax(info.zerr)) if info.zerr.size else float("nan")
        warnings.warn(f"{who} stopped at max_iter={cfg.max_iter} before its tolerance; the certified relative "
                      f"error of z is {worst:.3g}", ConvergenceWarning, stacklevel=3)
    return (z, info) if return_info else z


def tv_iso(x, gamma=1.0, *, ndim=2, weights=None, pixel_weights=None, tol=None, ztol=None, max_iter=1000,
           warm_start=None, return_info=False, deriv_tol=None, deriv_max_iter=10000, warn=True):
    """Isotropic TV prox of the last ``ndim`` axes of ``x``, differentiable in
    ``x``, ``gamma``, ``weights`` and ``pixel_weights`` (module docstring)."""
    return _device_tv(True, x, gamma, ndim, weights, pixel_weights, tol, ztol, max_iter, warm_start, return_info,
                      deriv_tol, deriv_max_iter, warn, "fastprox_b200.torch.tv_iso")


def tv_aniso(x, gamma=1.0, *, ndim=2, weights=None, edge_weights=None, tol=None, ztol=None, max_iter=1000,
             warm_start=None, return_info=False, deriv_tol=None, deriv_max_iter=10000, warn=True):
    """Anisotropic TV prox of the last ``ndim`` axes of ``x``, differentiable
    in ``x``, ``gamma``, ``weights`` and ``edge_weights``: the reverse pass
    averages the cotangent over the solution's constant components
    (tv_aniso.cpp:1398-1440)."""
    return _device_tv(False, x, gamma, ndim, weights, edge_weights, tol, ztol, max_iter, warm_start, return_info,
                      deriv_tol, deriv_max_iter, warn, "fastprox_b200.torch.tv_aniso")
