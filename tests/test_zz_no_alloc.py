"""fp_b200_tv_iso_noalloc: the isotropic solve for callers that cannot
allocate device memory (a custom operator inside a runtime with a fixed
memory plan, an allocator's out-of-memory handler, latency-bound code that
may not call cudaMalloc). It takes its scratch from a fixed array in the
library, so its results must match fp_prox's (which allocates a workspace)
call after call, with the array reused, up to the limits of that array; and
once the array is reserved on a device (the first call there), later calls
reserve no device memory at all. Collected last (file name), so a run that
stops at the first failure has run every other test first."""

import ctypes as C
import pathlib
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _noalloc(L, x, z, gamma, tol, max_iter, stream):
    B, H, W = x.shape
    gaps = np.zeros(B)
    iters = np.zeros(B, np.int32)
    st = L.fp_b200_tv_iso_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(z.data_ptr()), B, H, W, gamma, tol,
                                  max_iter, C.c_void_p(stream), gaps.ctypes.data_as(C.POINTER(C.c_double)),
                                  iters.ctypes.data_as(C.POINTER(C.c_int)))
    return st, gaps, iters


def _nrel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _against_fp_prox(cuda, cases, max_iter=2000):
    import torch

    from fastprox_b200 import TVIso, capi
    L = capi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for x_np, gamma in cases:
        x = torch.as_tensor(x_np, device=cuda)
        ref, info = TVIso(2).solve(x, gamma, tol=1e-6, max_iter=max_iter)
        z = torch.full_like(x, float("nan"))
        st, gaps, iters = _noalloc(L, x, z, gamma, 1e-6, max_iter, stream)
        assert st == (capi.FP_OK if info.converged else capi.FP_ENOTCONV)
        assert _nrel(z, ref) <= 1e-5  # the parity tolerance of the float32 tests
        assert np.array_equal(iters, info.image_iters), (iters, info.image_iters)
        np.testing.assert_allclose(gaps, info.gaps, rtol=1e-6)
        half = 0.5 * (x_np.astype(np.float64) ** 2).reshape(len(gaps), -1).sum(1)
        if info.converged:
            assert np.all(gaps <= 1e-6 * half)


def test_noalloc_matches_fp_prox_on_repeated_calls(cuda):
    from fastprox_b200 import synth
    _against_fp_prox(cuda, [(synth.phantom(3, 200, 256, seed=8), 0.1), (synth.phantom(3, 200, 256, seed=8), 0.1),
                            (synth.noise((2, 128, 96), 9), 0.2)])


def test_noalloc_at_its_limits(cuda):
    """Shapes at the edges of the scratch: one tall image (2048 rows of 512,
    one partial-sum slot per row), a narrow one (32768 x 32), the most images
    (64 x 128 x 128), and rows narrower than 32 pixels (the generic step)."""
    from fastprox_b200 import synth
    _against_fp_prox(cuda, [(synth.phantom(1, 2048, 512, seed=10), 0.1), (synth.phantom(1, 32768, 32, seed=11), 0.1),
                            (synth.phantom(64, 128, 128, seed=12), 0.1), (synth.phantom(4, 300, 20, seed=13), 0.1)],
                     max_iter=3000)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch

    from fastprox_b200 import capi
    L = capi.lib()
    x = torch.zeros(1, 8, 8, device=cuda)
    stream = torch.cuda.current_stream().cuda_stream
    big = L.fp_b200_tv_iso_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), 2, 1024, 1024, 0.1, 1e-6,
                                   10, C.c_void_p(stream), None, None)
    assert big == capi.FP_ESHAPE
    many = L.fp_b200_tv_iso_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), 65, 4, 4, 0.1, 1e-6, 10,
                                    C.c_void_p(stream), None, None)
    assert many == capi.FP_ESHAPE


_FRESH = r"""
import ctypes as C, sys
import torch
sys.path.insert(0, sys.argv[1])
from fastprox_b200 import capi, synth
L = capi.lib()
x = torch.as_tensor(synth.phantom(2, 96, 128, seed=3), device="cuda:0")
z = torch.empty_like(x)
s = torch.cuda.current_stream().cuda_stream
def call():
    return L.fp_b200_tv_iso_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(z.data_ptr()), 2, 96, 128, 0.1, 1e-6,
                                    2000, C.c_void_p(s), None, None)
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
assert call() == capi.FP_OK  # the warm-up call: reserves the array on this device
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
for _ in range(3):
    assert call() == capi.FP_OK
torch.cuda.synchronize()
free2 = torch.cuda.mem_get_info()[0]
print(free0, free1, free2)
assert free2 == free1, (free0, free1, free2)
"""


def test_noalloc_reserves_nothing_after_the_first_call(cuda):
    """In a fresh process: the first call on the device may reserve the
    library's module with its scratch array; later calls leave the device's
    free memory unchanged."""
    r = subprocess.run([sys.executable, "-c", _FRESH, str(ROOT)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr[-3000:]
