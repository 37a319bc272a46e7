"""ctypes bindings to libfastprox_b200.so (the C ABI of include/fastprox_b200.h).

The library is loaded from this package's directory only; a missing or
unloadable library raises at import of the functions that need it. There is
no fallback of any kind.
"""

from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libfastprox_b200.so"

FP_F32, FP_F64, FP_I8, FP_I32, FP_I64 = 1, 2, 3, 4, 5
FP_DEVICE_CPU, FP_DEVICE_CUDA = 0, 2
STATUS = ["FP_OK", "FP_EINVAL", "FP_EDTYPE", "FP_ESHAPE", "FP_ENOMEM", "FP_ENOTCONV", "FP_EPARAM",
          "FP_EINTERNAL", "FP_EDEVICE"]
FP_OK, FP_EINVAL, FP_EDTYPE, FP_ESHAPE, FP_ENOMEM, FP_ENOTCONV, FP_EPARAM, FP_EINTERNAL, FP_EDEVICE = range(9)


class FpArray(C.Structure):
    _fields_ = [("data", C.c_void_p), ("dtype", C.c_int), ("ndim", C.c_int),
                ("shape", C.POINTER(C.c_int64)), ("strides", C.POINTER(C.c_int64)),
                ("device", C.c_int)]


class FpOptions(C.Structure):
    _fields_ = [("axis", C.c_int), ("threads", C.c_int), ("tol", C.c_double),
                ("max_iter", C.c_int), ("tie", C.c_int), ("keep_structure", C.c_int)]


class FpInfo(C.Structure):
    _fields_ = [("gap", C.c_double), ("iters", C.c_int), ("ties", C.c_int64)]


class FastproxError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        name = STATUS[status] if 0 <= status < len(STATUS) else str(status)
        super().__init__(f"{what}: {name}")


_lib = None

# name -> (restype, argtypes); the declarations of include/fastprox_b200.h
_P = C.c_void_p
_A = C.POINTER(FpArray)
SIGNATURES = {
    "fp_options_init": (None, [C.POINTER(FpOptions)]),
    "fp_op_tv_iso": (C.c_int, [C.c_int, _A, C.POINTER(_P)]),
    "fp_op_tv_aniso": (C.c_int, [C.c_int, _A, C.POINTER(_P)]),
    "fp_op_tv_iso_weighted": (C.c_int, [C.c_int, _A, _A, C.POINTER(_P)]),
    "fp_op_tv_aniso_weighted": (C.c_int, [C.c_int, _A, _A, C.POINTER(_P)]),
    "fp_op_free": (None, [_P]),
    "fp_op_nparams": (C.c_int64, [_P]),
    "fp_op_name": (C.c_char_p, [_P]),
    "fp_workspace_create": (C.c_int, [_P, _A, C.POINTER(FpOptions), C.POINTER(_P)]),
    "fp_workspace_free": (None, [_P]),
    "fp_workspace_get_dual": (C.c_int, [_P, _A]),
    "fp_workspace_set_dual": (C.c_int, [_P, _A]),
    "fp_workspace_set_warm": (C.c_int, [_P, C.c_int]),
    "fp_workspace_set_deriv_tol": (C.c_int, [_P, C.c_double, C.c_int]),
    "fp_workspace_deriv_info": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "fp_prox": (C.c_int, [_P, C.c_double, _A, _A, C.POINTER(FpOptions), _P, C.POINTER(FpInfo)]),
    "fp_prox_steps": (C.c_int, [_P, _A, _A, _A, C.POINTER(FpOptions), _P]),
    "fp_prox_conj": (C.c_int, [_P, C.c_double, _A, _A, C.POINTER(FpOptions), _P, C.POINTER(FpInfo)]),
    "fp_jvp": (C.c_int, [_P, _P, _A, C.c_double, _A, _A]),
    "fp_vjp": (C.c_int, [_P, _P, _A, _A, C.POINTER(C.c_double), _A]),
    "fp_vjp_device": (C.c_int, [_P, _P, _A, _A, _A, _A]),
    "fp_workspace_kinks": (C.c_int, [_P, C.c_double, _A, C.POINTER(C.c_int64)]),
    "fp_workspace_set_branch": (C.c_int, [_P, _A, C.c_double]),
    "fp_op_struct_kind": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "fp_workspace_units": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "fp_workspace_states": (C.c_int, [_P, _A, C.POINTER(C.c_int64)]),
    "fp_workspace_regions": (C.c_int, [_P, _A, _A, C.POINTER(C.c_int64), C.c_int64]),
    "fp_workspace_constraint": (C.c_int, [_P, _A, C.POINTER(C.c_int8), C.c_int64]),
    "fp_workspace_deriv_exact": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "fp_workspace_refine": (C.c_int, [_P, _P, C.c_double, C.c_int, _A, C.POINTER(FpInfo)]),
    "fp_device_available": (C.c_int, [C.c_int]),
    "fp_op_device_check": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "fp_workspace_set_stream": (C.c_int, [_P, _P]),
    "fp_workspace_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "fp_workspace_info": (C.c_int, [_P, C.POINTER(FpInfo)]),
    "fp_workspace_image_info": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                          C.POINTER(C.c_double), C.c_int64]),
    "fp_strerror": (C.c_char_p, [C.c_int]),
    "fp_abi_version": (C.c_int, []),
    "fp_version_string": (C.c_char_p, []),
    "fp_default_threads": (C.c_int, []),
    "fp_b200_workspace_stats": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "fp_b200_workspace_time_steps": (C.c_int, [_P, C.c_int]),
    "fp_b200_workspace_step_times": (C.c_int, [_P, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "fp_b200_release_cached": (None, []),
    "fp_b200_batch_create": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int, C.POINTER(_P)]),
    "fp_b200_batch_free": (None, [_P]),
    "fp_b200_batch_set_stream": (C.c_int, [_P, _P]),
    "fp_b200_batch_set_rows": (C.c_int, [_P, C.c_int]),
    "fp_b200_batch_set_graphs": (C.c_int, [_P, C.c_int]),
    "fp_b200_batch_admit": (C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int, _P,
                                      C.POINTER(C.c_int)]),
    "fp_b200_batch_run": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fp_b200_batch_stats": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "fp_b200_op_tv_iso_huber": (C.c_int, [C.c_int, _A, _A, C.c_double, C.POINTER(_P)]),
    "fp_b200_op_tv_aniso_huber": (C.c_int, [C.c_int, _A, _A, C.c_double, C.POINTER(_P)]),
    "fp_b200_batch_set_quads": (C.c_int, [_P, C.c_int, C.c_int]),
    "fp_b200_vjp_images": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64]),
    "fp_b200_tv_iso_noalloc": (C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int,
                                         _P, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
}


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `python -m fastprox_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, what, ok=(FP_OK,)):
    if status not in ok:
        raise FastproxError(status, what)
    return status


class ArrayRef:
    """An fp_array describing a NumPy array or a torch tensor (CPU or CUDA),
    keeping its shape and stride buffers alive."""

    def __init__(self, a):
        if isinstance(a, np.ndarray):
            dt = {np.dtype(np.float32): FP_F32, np.dtype(np.float64): FP_F64, np.dtype(np.int8): FP_I8,
                  np.dtype(np.int32): FP_I32, np.dtype(np.int64): FP_I64}[a.dtype]
            shape, strides = a.shape, tuple(s // a.itemsize for s in a.strides)
            ptr, dev = a.ctypes.data, FP_DEVICE_CPU
        else:  # torch.Tensor
            import torch
            dt = {torch.float32: FP_F32, torch.float64: FP_F64, torch.int8: FP_I8, torch.int32: FP_I32,
                  torch.int64: FP_I64}[a.dtype]
            shape, strides = tuple(a.shape), tuple(a.stride())
            ptr = a.data_ptr()
            dev = FP_DEVICE_CUDA if a.is_cuda else FP_DEVICE_CPU
        self.obj = a
        n = max(1, len(shape))
        self.shape = (C.c_int64 * n)(*shape)
        self.strides = (C.c_int64 * n)(*strides)
        self.s = FpArray(ptr, dt, len(shape), self.shape, self.strides, dev)

    def ref(self):
        return C.byref(self.s)


def options(tol=1e-6, max_iter=1000, keep=False):
    o = FpOptions()
    lib().fp_options_init(C.byref(o))
    o.tol, o.max_iter, o.keep_structure = float(tol), int(max_iter), int(bool(keep))
    return o
