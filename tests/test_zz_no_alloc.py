"""fp_b200_tv_iso_noalloc: the isotropic solve for callers that cannot
allocate device memory (a custom operator inside a runtime with a fixed
memory plan, an allocator's out-of-memory handler, latency-bound code that
may not call cudaMalloc). It takes its scratch from a fixed array in the
library, so its results must match fp_prox's (which allocates a workspace)
call after call, with the array reused. Collected last (file name), so a
run that stops at the first failure has run every other test first."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


def test_noalloc_matches_fp_prox_on_repeated_calls(cuda):
    import torch

    from fastprox_b200 import TVIso, capi, synth
    L = capi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(synth.phantom(3, 200, 256, seed=8), 0.1), (synth.phantom(3, 200, 256, seed=8), 0.1),
             (synth.noise((2, 128, 96), 9), 0.2)]
    for x_np, gamma in cases:
        x = torch.as_tensor(x_np, device=cuda)
        ref, info = TVIso(2).solve(x, gamma, tol=1e-6, max_iter=2000)
        z = torch.full_like(x, float("nan"))
        st, gaps, iters = _noalloc(L, x, z, gamma, 1e-6, 2000, stream)
        assert st == capi.FP_OK
        assert _nrel(z, ref) <= 1e-5  # the parity tolerance of the float32 tests
        assert np.array_equal(iters, info.image_iters)
        np.testing.assert_allclose(gaps, info.gaps, rtol=1e-6)


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
