"""Operator objects over the C ABI: the host-side mirror of the reference's
``fastprox.TVIso`` / ``fastprox.TVAniso`` (bindings/python/fastprox/__init__.py)
for the image-TV path.

``TVIso(ndim, weights, pixel_weights)`` and ``TVAniso(ndim, weights,
edge_weights)`` build the operator once (``fp_op_tv_iso[_weighted]``,
``fp_op_tv_aniso[_weighted]``); ``prox`` / ``solve`` run ``fp_prox`` (or
``fp_prox_steps`` for one step per image) on NumPy arrays (staged through the
GPU) or torch tensors (CUDA: solved in place on the tensor's device and
current stream). Workspaces are cached per (shape, dtype, device).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import capi


@dataclass
class IterInfo:
    """Results of one call (the reference's IterInfo, __init__.py:97-122):
    gap = sum of the per-image gaps, iters = their max, converged = every
    image met tol; per-image gaps, iterations and certified relative errors
    of z; the dual (ndim, *x.shape) in the reference's form."""
    gap: float
    iters: int
    converged: bool
    gaps: np.ndarray = field(default=None)
    image_iters: np.ndarray = field(default=None)
    zerr: np.ndarray = field(default=None)
    dual: object = None


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _is_scalar(g):
    if isinstance(g, (int, float)):
        return True
    if _is_torch(g):
        return g.dim() == 0
    return np.ndim(g) == 0


class _ImageOp:
    iso = True
    delta = None  # Huber-smoothed TV: its smoothing delta

    def __init__(self, ndim=2, weights=None, spatial=None):
        L = capi.lib()
        self.k = int(ndim)
        self._op = C.c_void_p()
        w = None if weights is None else np.ascontiguousarray(np.atleast_1d(np.asarray(weights, np.float64)))
        wref = None if w is None else capi.ArrayRef(w)
        if self.delta is not None:
            sp = None if spatial is None else capi.ArrayRef(np.ascontiguousarray(np.asarray(spatial, np.float64)))
            f = L.fp_b200_op_tv_iso_huber if self.iso else L.fp_b200_op_tv_aniso_huber
            st = f(self.k, None if wref is None else wref.ref(), None if sp is None else sp.ref(), float(self.delta),
                   C.byref(self._op))
        elif spatial is None:
            f = L.fp_op_tv_iso if self.iso else L.fp_op_tv_aniso
            st = f(self.k, None if wref is None else wref.ref(), C.byref(self._op))
        else:
            sp = np.ascontiguousarray(np.asarray(spatial, np.float64))
            f = L.fp_op_tv_iso_weighted if self.iso else L.fp_op_tv_aniso_weighted
            st = f(self.k, None if wref is None else wref.ref(), capi.ArrayRef(sp).ref(), C.byref(self._op))
        capi.check(st, "operator")
        self._ws = {}

    def __del__(self):
        try:
            L = capi.lib()
            for ws in self._ws.values():
                L.fp_workspace_free(ws)
            if self._op:
                L.fp_op_free(self._op)
        except Exception:
            pass

    def release(self):
        """Frees the cached workspaces (created again on the next solve): for
        callers that solve many shapes with one operator."""
        L = capi.lib()
        for ws in self._ws.values():
            L.fp_workspace_free(ws)
        self._ws.clear()

    @property
    def nparams(self):
        return int(capi.lib().fp_op_nparams(self._op))

    def workspace(self, x, keep=False):
        """The cached workspace for x's shape, dtype and device."""
        if _is_torch(x):
            key = (tuple(x.shape), str(x.dtype), str(x.device), keep)
        else:
            key = (tuple(x.shape), str(x.dtype), "cpu", keep)
        ws = self._ws.get(key)
        if ws is None:
            ws = C.c_void_p()
            opt = capi.options(keep=keep)
            capi.check(capi.lib().fp_workspace_create(self._op, capi.ArrayRef(x).ref(), C.byref(opt),
                                                      C.byref(ws)), "workspace")
            self._ws[key] = ws
        return ws

    def solve(self, x, gamma=1.0, *, tol=1e-6, max_iter=1000, out=None, warm=False, dual=None,
              with_dual=True, warn=False):
        """z = prox_{gamma g}(x) and an IterInfo. gamma: a number, or one
        step per image (an array or tensor of x's batch shape). FP_ENOTCONV
        is reported through info.converged; other errors raise."""
        L = capi.lib()
        torch_mode = _is_torch(x)
        if torch_mode:
            import torch
            if out is None:
                out = torch.empty_like(x, memory_format=torch.contiguous_format)
        else:
            x = np.asarray(x)
            if out is None:
                out = np.empty(x.shape, x.dtype)
        ws = self.workspace(x)
        if torch_mode and x.is_cuda:
            import torch
            with torch.cuda.device(x.device):
                stream = torch.cuda.current_stream().cuda_stream
            capi.check(L.fp_workspace_set_stream(ws, C.c_void_p(stream)), "set_stream")
        capi.check(L.fp_workspace_set_warm(ws, int(bool(warm))), "set_warm")
        if dual is not None:
            capi.check(L.fp_workspace_set_dual(ws, capi.ArrayRef(dual).ref()), "set_dual")
        opt = capi.options(tol=tol, max_iter=max_iter)
        xr, orf = capi.ArrayRef(x), capi.ArrayRef(out)
        ok = (capi.FP_OK, capi.FP_ENOTCONV)
        if _is_scalar(gamma):
            info = capi.FpInfo()
            st = L.fp_prox(self._op, float(gamma), xr.ref(), orf.ref(), C.byref(opt), ws, C.byref(info))
        else:
            st = L.fp_prox_steps(self._op, capi.ArrayRef(gamma).ref(), xr.ref(), orf.ref(), C.byref(opt), ws)
        capi.check(st, "fp_prox", ok)
        B = int(np.prod(x.shape[: x.ndim - self.k], dtype=np.int64)) if x.ndim > self.k else 1
        gaps = np.zeros(B)
        its = np.zeros(B, np.int32)
        zerr = np.zeros(B)
        capi.check(L.fp_workspace_image_info(ws, gaps.ctypes.data_as(C.POINTER(C.c_double)),
                                             its.ctypes.data_as(C.POINTER(C.c_int)),
                                             zerr.ctypes.data_as(C.POINTER(C.c_double)), B), "image_info")
        d = None
        if with_dual:
            if torch_mode:
                import torch
                d = torch.empty((self.k,) + tuple(x.shape), dtype=x.dtype, device=x.device)
            else:
                d = np.empty((self.k,) + x.shape, x.dtype)
            capi.check(L.fp_workspace_get_dual(ws, capi.ArrayRef(d).ref()), "get_dual")
        info = IterInfo(float(np.nansum(gaps)) if not np.isnan(gaps).all() else float("nan"),
                        int(its.max(initial=0)), st == capi.FP_OK, gaps, its, zerr, d)
        return out, info

    def prox(self, x, gamma=1.0, **kw):
        return self.solve(x, gamma, with_dual=False, **kw)[0]


class TVIso(_ImageOp):
    """Isotropic TV: gamma sum_p alpha_p |(w_0 D_0 z, ..., w_{k-1} D_{k-1} z)_p|_2."""
    iso = True

    def __init__(self, ndim=2, weights=None, pixel_weights=None):
        super().__init__(ndim, weights, pixel_weights)


class TVAniso(_ImageOp):
    """Anisotropic TV: gamma sum_a w_a sum_p beta_{a,p} |z_{p+e_a} - z_p|."""
    iso = False

    def __init__(self, ndim=2, weights=None, edge_weights=None):
        super().__init__(ndim, weights, edge_weights)


class TVIsoHuber(_ImageOp):
    """Huber-smoothed isotropic TV: gamma sum_p alpha_p h_delta(|(W D z)_p|)."""
    iso = True

    def __init__(self, ndim=2, weights=None, pixel_weights=None, delta=1e-2):
        self.delta = float(delta)
        super().__init__(ndim, weights, pixel_weights)


class TVAnisoHuber(_ImageOp):
    """Huber-smoothed anisotropic TV: gamma sum_{a,p} beta_{a,p} h_delta(|w_a (D_a z)_p|)."""
    iso = False

    def __init__(self, ndim=2, weights=None, edge_weights=None, delta=1e-2):
        self.delta = float(delta)
        super().__init__(ndim, weights, edge_weights)


def tv_iso(x, gamma=1.0, *, ndim=2, weights=None, pixel_weights=None, **kw):
    return TVIso(ndim, weights, pixel_weights).solve(x, gamma, **kw)


def tv_aniso(x, gamma=1.0, *, ndim=2, weights=None, edge_weights=None, **kw):
    return TVAniso(ndim, weights, edge_weights).solve(x, gamma, **kw)
