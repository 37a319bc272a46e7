"""ctypes bindings to the reference fastprox C library (test infrastructure).

The library is built from the reference's own sources by ``oracle/Makefile``
into ``oracle/_ref/libfastprox_ref.so``; nothing here is product code. The
structures restate the public ABI of ``include/fastprox.h:52-109`` (fp_dtype,
fp_device, fp_array, fp_status, fp_options, fp_info) so that the calls
below are exactly those a C user of the reference makes.
"""

from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libfastprox_ref.so"

FP_F32, FP_F64 = 1, 2
FP_OK, FP_ENOTCONV = 0, 5


class FpArray(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int), ("ndim", C.c_int),
                ("shape", C.POINTER(C.c_int64)), ("strides", C.POINTER(C.c_int64)),
                ("device", C.c_int)]


class FpOptions(C.Structure):
    _fields_ = [("axis", C.c_int), ("threads", C.c_int), ("tol", C.c_double),
                ("max_iter", C.c_int), ("tie", C.c_int), ("keep_structure", C.c_int)]


class FpInfo(C.Structure):
    _fields_ = [("gap", C.c_double), ("iters", C.c_int), ("ties", C.c_int64)]


_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is not built (make -C oracle)")
        L = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        L.fp_options_init.argtypes = [C.POINTER(FpOptions)]
        for name in ("fp_op_tv_iso", "fp_op_tv_aniso"):
            getattr(L, name).argtypes = [C.c_int, C.POINTER(FpArray), C.POINTER(P)]
        for name in ("fp_op_tv_iso_weighted", "fp_op_tv_aniso_weighted"):
            getattr(L, name).argtypes = [C.c_int, C.POINTER(FpArray), C.POINTER(FpArray), C.POINTER(P)]
        L.fp_op_free.argtypes = [P]
        L.fp_workspace_create.argtypes = [P, C.POINTER(FpArray), C.POINTER(FpOptions), C.POINTER(P)]
        L.fp_workspace_free.argtypes = [P]
        L.fp_prox.argtypes = [P, C.c_double, C.POINTER(FpArray), C.POINTER(FpArray), C.POINTER(FpOptions), P,
                              C.POINTER(FpInfo)]
        L.fp_prox_steps.argtypes = [P, C.POINTER(FpArray), C.POINTER(FpArray), C.POINTER(FpArray),
                                    C.POINTER(FpOptions), P]
        L.fp_prox_conj.argtypes = [P, C.c_double, C.POINTER(FpArray), C.POINTER(FpArray), C.POINTER(FpOptions), P,
                                   C.POINTER(FpInfo)]
        L.fp_workspace_image_info.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                              C.POINTER(C.c_double), C.c_int64]
        L.fp_workspace_get_dual.argtypes = [P, C.POINTER(FpArray)]
        L.fp_workspace_set_dual.argtypes = [P, C.POINTER(FpArray)]
        L.fp_workspace_set_warm.argtypes = [P, C.c_int]
        L.fp_vjp.argtypes = [P, P, C.POINTER(FpArray), C.POINTER(FpArray), C.POINTER(C.c_double),
                             C.POINTER(FpArray)]
        L.fp_jvp.argtypes = [P, P, C.POINTER(FpArray), C.c_double, C.POINTER(FpArray), C.POINTER(FpArray)]
        L.fp_workspace_set_deriv_tol.argtypes = [P, C.c_double, C.c_int]
        L.fp_workspace_regions.argtypes = [P, C.POINTER(FpArray), C.POINTER(FpArray), C.POINTER(C.c_int64),
                                           C.c_int64]
        L.fp_workspace_kinks.argtypes = [P, C.c_double, C.POINTER(FpArray), C.POINTER(C.c_int64)]
        L.fp_workspace_set_branch.argtypes = [P, C.POINTER(FpArray), C.c_double]
        L.fp_workspace_deriv_exact.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.fp_workspace_deriv_info.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.fp_strerror.restype = C.c_char_p
        _lib = L
    return _lib


class _Arr:
    """An fp_array view of a NumPy array (kept alive with its shape buffer)."""

    def __init__(self, a: np.ndarray):
        self.a = a
        self.shape = (C.c_int64 * max(1, a.ndim))(*a.shape)
        self.strides = (C.c_int64 * max(1, a.ndim))(*[s // a.itemsize for s in a.strides])
        dt = {np.dtype(np.float32): FP_F32, np.dtype(np.float64): FP_F64, np.dtype(np.int8): 3,
              np.dtype(np.int32): 4, np.dtype(np.int64): 5}[a.dtype]
        self.s = FpArray(a.ctypes.data, dt, a.ndim, self.shape, self.strides, 0)

    def ref(self):
        return C.byref(self.s)


def _check(status, what):
    if status not in (FP_OK, FP_ENOTCONV):
        raise RuntimeError(f"{what}: {lib().fp_strerror(status).decode()} ({status})")
    return status


def make_op(iso: bool, k: int, w=None, spatial=None):
    """fp_op_tv_iso / fp_op_tv_aniso (``_weighted`` with pixel or edge weights)."""
    L = lib()
    op = C.c_void_p()
    wa = None if w is None else _Arr(np.ascontiguousarray(np.atleast_1d(np.asarray(w, np.float64))))
    wref = None if wa is None else wa.ref()
    if spatial is None:
        st = (L.fp_op_tv_iso if iso else L.fp_op_tv_aniso)(k, wref, C.byref(op))
    else:
        sa = _Arr(np.ascontiguousarray(np.asarray(spatial, np.float64)))
        st = (L.fp_op_tv_iso_weighted if iso else L.fp_op_tv_aniso_weighted)(k, wref, sa.ref(), C.byref(op))
    _check(st, "make_op")
    return op


class Result:
    def __init__(self, z, gaps, iters, zerrs, dual, status):
        self.z, self.gaps, self.iters, self.zerrs, self.dual, self.status = z, gaps, iters, zerrs, dual, status

    @property
    def converged(self):
        return self.status == FP_OK


def solve(x, gamma, *, iso=True, k=2, w=None, spatial=None, tol=1e-6, max_iter=1000, threads=0,
          steps=None, warm_dual=None, keep=False, conj=False):
    """One reference call on x (batch over leading axes, images the last k).

    ``gamma`` is one step, or ``steps`` one per image (``fp_prox_steps``);
    with ``conj`` the call is ``fp_prox_conj`` and ``gamma`` its sigma.
    Returns a Result with z (x's dtype), per-image gaps/iters/zerrs and the
    dual (k, *x.shape) in float64, the reference's own form."""
    L = lib()
    x = np.ascontiguousarray(x)
    op = make_op(iso, k, w, spatial)
    opt = FpOptions()
    L.fp_options_init(C.byref(opt))
    opt.tol, opt.max_iter, opt.threads, opt.keep_structure = float(tol), int(max_iter), int(threads), int(keep)
    xa = _Arr(x)
    ws = C.c_void_p()
    _check(L.fp_workspace_create(op, xa.ref(), C.byref(opt), C.byref(ws)), "workspace")
    try:
        if warm_dual is not None:
            da = _Arr(np.ascontiguousarray(warm_dual, np.float64))
            _check(L.fp_workspace_set_dual(ws, da.ref()), "set_dual")
        z = np.empty_like(x)
        za = _Arr(z)
        if conj:
            info = FpInfo()
            st = L.fp_prox_conj(op, float(gamma), xa.ref(), za.ref(), C.byref(opt), ws, C.byref(info))
        elif steps is None:
            info = FpInfo()
            st = L.fp_prox(op, float(gamma), xa.ref(), za.ref(), C.byref(opt), ws, C.byref(info))
        else:
            sa = _Arr(np.ascontiguousarray(np.asarray(steps, np.float64).reshape(x.shape[:x.ndim - k])))
            st = L.fp_prox_steps(op, sa.ref(), xa.ref(), za.ref(), C.byref(opt), ws)
        _check(st, "fp_prox")
        B = int(np.prod(x.shape[:x.ndim - k], dtype=np.int64))
        gaps = np.zeros(B)
        iters = np.zeros(B, np.int32)
        zerrs = np.zeros(B)
        _check(L.fp_workspace_image_info(ws, gaps.ctypes.data_as(C.POINTER(C.c_double)),
                                         iters.ctypes.data_as(C.POINTER(C.c_int)),
                                         zerrs.ctypes.data_as(C.POINTER(C.c_double)), B), "image_info")
        dual = None
        if not conj:  # the reference keeps no dual of a conjugate call
            dual = np.empty((k,) + x.shape, np.float64)
            _check(L.fp_workspace_get_dual(ws, _Arr(dual).ref()), "get_dual")
        res = Result(z, gaps, iters, zerrs, dual, st)
        if keep:
            res._ws, res._op = ws, op
            ws = None
            op = None
        return res
    finally:
        if ws is not None:
            L.fp_workspace_free(ws)
        if op is not None:
            L.fp_op_free(op)


def vjp(res: Result, g, nparams: int, deriv_tol=None):
    """fp_vjp at a kept Result: (gx, ggamma, gparams); deriv_tol sets the
    derivative's solve tolerance first (fp_workspace_set_deriv_tol)."""
    L = lib()
    if deriv_tol is not None:
        _check(L.fp_workspace_set_deriv_tol(res._ws, float(deriv_tol), 1000000), "deriv_tol")
    g = np.ascontiguousarray(g, res.z.dtype)
    gx = np.empty_like(g)
    gp = np.zeros(nparams, np.float64)
    ga, gxa, gpa = _Arr(g), _Arr(gx), _Arr(gp)
    gg = C.c_double(0.0)
    _check(L.fp_vjp(res._op, res._ws, ga.ref(), gxa.ref(), C.byref(gg), gpa.ref()), "fp_vjp")
    return gx, gg.value, gp


def jvp(res: Result, dx, dgamma: float, dparams=None):
    """fp_jvp at a kept Result: dz for the direction (dx, dgamma, dparams);
    dx or dparams None reads as zero."""
    L = lib()
    dz = np.empty_like(res.z)
    dxa = None if dx is None else _Arr(np.ascontiguousarray(dx, res.z.dtype))
    dpa = None if dparams is None else _Arr(np.ascontiguousarray(dparams, np.float64))
    _check(L.fp_jvp(res._op, res._ws, None if dxa is None else dxa.ref(), float(dgamma),
                    None if dpa is None else dpa.ref(), _Arr(dz).ref()), "fp_jvp")
    return dz


def regions(res: Result, nimages: int):
    """fp_workspace_regions at a kept Result: (labels int64, nregions)."""
    L = lib()
    lab = np.empty(res.z.shape, np.int64)
    nreg = (C.c_int64 * nimages)()
    _check(L.fp_workspace_regions(res._ws, _Arr(lab).ref(), None, nreg, nimages), "regions")
    return lab, np.array(list(nreg), np.int64)


def kinks(res: Result, tol: float):
    """fp_workspace_kinks at a kept Result: (mask int8, count)."""
    L = lib()
    m = np.empty(res.z.shape, np.int8)
    c = C.c_int64()
    _check(L.fp_workspace_kinks(res._ws, float(tol), _Arr(m).ref(), C.byref(c)), "kinks")
    return m, c.value


def set_branch(res: Result, side, tol: float):
    L = lib()
    sa = None if side is None else _Arr(np.ascontiguousarray(side, np.int8))
    _check(L.fp_workspace_set_branch(res._ws, None if sa is None else sa.ref(), float(tol)), "set_branch")


def deriv_exact(res: Result):
    L = lib()
    ex, mu = C.c_int(), C.c_double()
    _check(L.fp_workspace_deriv_exact(res._ws, C.byref(ex), C.byref(mu)), "deriv_exact")
    return ex.value, mu.value


def release(res: Result):
    L = lib()
    if getattr(res, "_ws", None) is not None:
        L.fp_workspace_free(res._ws)
        L.fp_op_free(res._op)
        res._ws = res._op = None


def default_threads() -> int:
    return len(os.sched_getaffinity(0))
