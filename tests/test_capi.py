"""The C-ABI library without a GPU: it loads, exports every entry point
include/fastprox_b200.h declares, lays out the ABI structures as the
reference's fastprox.h does, and rejects bad arguments before touching a
device (no compute call here)."""

import ctypes as C
import pathlib
import re

import numpy as np
import pytest

from fastprox_b200 import capi

HEADER = pathlib.Path(__file__).resolve().parents[1] / "include" / "fastprox_b200.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"FP_API[^;(]*?\b(fp_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    L = capi.lib()
    names = declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(capi.SIGNATURES), set(names) ^ set(capi.SIGNATURES)


def test_abi_layout_matches_reference_header():
    # fastprox.h:61-68, 93-109 on LP64
    assert C.sizeof(capi.FpArray) == 40
    assert C.sizeof(capi.FpOptions) == 32
    assert C.sizeof(capi.FpInfo) == 24
    L = capi.lib()
    assert L.fp_abi_version() == 1
    assert L.fp_strerror(capi.FP_ENOTCONV) == b"iterative operator did not converge"


def test_options_defaults():
    o = capi.options()
    assert (o.axis, o.threads, o.max_iter, o.tie, o.keep_structure) == (-1, 0, 1000, 0, 0)
    assert o.tol == 1e-6


def _op(fn, *args):
    op = C.c_void_p()
    st = fn(*args, C.byref(op))
    return st, op


def test_operator_parameter_errors():
    L = capi.lib()
    assert _op(L.fp_op_tv_iso, 4, None)[0] == capi.FP_EPARAM
    assert _op(L.fp_op_tv_aniso, 1, None)[0] == capi.FP_EPARAM
    w = capi.ArrayRef(np.array([1.0, -1.0]))
    assert _op(L.fp_op_tv_iso, 2, w.ref())[0] == capi.FP_EPARAM
    w3 = capi.ArrayRef(np.array([1.0, 1.0, 1.0]))
    assert _op(L.fp_op_tv_iso, 2, w3.ref())[0] == capi.FP_ESHAPE
    al = capi.ArrayRef(np.full((4, 5), np.nan))
    assert _op(L.fp_op_tv_iso_weighted, 2, None, al.ref())[0] == capi.FP_EPARAM
    be = capi.ArrayRef(np.ones((3, 4, 5)))
    assert _op(L.fp_op_tv_aniso_weighted, 2, None, be.ref())[0] == capi.FP_ESHAPE
    st, op = _op(L.fp_op_tv_iso_weighted, 2, capi.ArrayRef(np.array([2.0])).ref(),
                 capi.ArrayRef(np.ones((4, 5))).ref())
    assert st == capi.FP_OK
    assert L.fp_op_nparams(op) == 2 + 20 and L.fp_op_name(op) == b"tv_iso"
    L.fp_op_free(op)
    st, op = _op(L.fp_op_tv_aniso, 3, None)
    assert st == capi.FP_OK and L.fp_op_nparams(op) == 3 and L.fp_op_name(op) == b"tv_aniso"
    L.fp_op_free(op)


def test_prox_argument_errors_before_any_device_work():
    L = capi.lib()
    st, op = _op(L.fp_op_tv_iso, 2, None)
    x = np.zeros((2, 8, 8), np.float32)
    out = np.zeros((2, 8, 8), np.float32)
    o64 = np.zeros((2, 8, 8), np.float64)
    opt = capi.options()
    xr, orf = capi.ArrayRef(x), capi.ArrayRef(out)
    assert L.fp_prox(op, -1.0, xr.ref(), orf.ref(), None, None, None) == capi.FP_EPARAM
    assert L.fp_prox(op, float("inf"), xr.ref(), orf.ref(), None, None, None) == capi.FP_EPARAM
    assert L.fp_prox(op, 0.1, xr.ref(), capi.ArrayRef(o64).ref(), None, None, None) == capi.FP_EDTYPE
    assert L.fp_prox(op, 0.1, xr.ref(), capi.ArrayRef(out[:1]).ref(), None, None, None) == capi.FP_ESHAPE
    bad = capi.options(max_iter=0)
    assert L.fp_prox(op, 0.1, xr.ref(), orf.ref(), C.byref(bad), None, None) == capi.FP_EPARAM
    keep = capi.options(keep=True)
    assert L.fp_prox(op, 0.1, xr.ref(), orf.ref(), C.byref(keep), None, None) == capi.FP_EINVAL
    # partial overlap of out with x (not the same view)
    big = np.zeros((3, 8, 8), np.float32)
    a, b = capi.ArrayRef(big[:2]), capi.ArrayRef(big[1:])
    assert L.fp_prox(op, 0.1, a.ref(), b.ref(), None, None, None) == capi.FP_EINVAL
    # a 1-d array has fewer axes than the image
    v = capi.ArrayRef(np.zeros(5, np.float32))
    assert L.fp_prox(op, 0.1, v.ref(), capi.ArrayRef(np.zeros(5, np.float32)).ref(), None, None, None) \
        == capi.FP_ESHAPE
    # an empty batch is fine and does nothing
    e = np.zeros((0, 8, 8), np.float32)
    assert L.fp_prox(op, 0.1, capi.ArrayRef(e).ref(), capi.ArrayRef(e.copy()).ref(), C.byref(opt), None,
                     None) == capi.FP_OK
    L.fp_op_free(op)


def test_no_gpu_means_device_error_not_a_cpu_fallback():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    L = capi.lib()
    assert L.fp_device_available(capi.FP_DEVICE_CUDA) == 0
    st, op = _op(L.fp_op_tv_iso, 2, None)
    x = np.ones((1, 8, 8), np.float32)
    out = np.zeros_like(x)
    assert L.fp_prox(op, 0.1, capi.ArrayRef(x).ref(), capi.ArrayRef(out).ref(), None, None, None) \
        == capi.FP_EDEVICE
    assert not out.any()
    ws = C.c_void_p()
    assert L.fp_workspace_create(op, capi.ArrayRef(x).ref(), None, C.byref(ws)) == capi.FP_EDEVICE
    L.fp_op_free(op)
