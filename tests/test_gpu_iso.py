"""Isotropic TV on the GPU against the reference (the parity tests proper).

Every call goes through the C ABI (libfastprox_b200.so) on CUDA tensors or
on host arrays staged through the GPU. The checks are the reference's own
outputs on the same seeded inputs (tests/golden/ref_vectors.npz), the
oracle at the 8 x 256^2 workload, the certificate, and the edge cases the
reference tests (NaN and Inf images, zero steps, single active axis,
max_iter, strided arrays, warm starts, conjugates).

Tolerances: float32 z within 1e-5 of the reference relative to 1 + max|x|
(FP32 iterates against the reference's FP64 ones); float64 within 1e-9.
Iteration counts equal (float64) or within one gap-check period (float32).
"""

import numpy as np
import pytest

from golden_data import ref_vectors

pytestmark = pytest.mark.gpu

REF = ref_vectors()
ISO = sorted(n for n, c in REF.items() if int(c["iso"]) == 1)
TOL32, TOL64 = 1e-5, 1e-9


def _torch():
    import torch
    return torch


def _solve(c, x, **kw):
    from fastprox_b200 import TVIso
    op = TVIso(int(c["k"]), c.get("weights"), c.get("spatial"))
    gamma = c["steps"] if "steps" in c else float(c["gamma"])
    if "steps" in c and not isinstance(x, np.ndarray):
        gamma = _torch().as_tensor(c["steps"], device=x.device)
    return op.solve(x, gamma, tol=float(c["tol"]), max_iter=int(c["max_iter"]), **kw)


def _rel(a, b, x):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() / (1 + np.abs(x).max()))


@pytest.mark.parametrize("name", ISO)
def test_matches_reference_vectors_device(cuda, name):
    torch = _torch()
    c = REF[name]
    x = c["x"]
    xt = torch.as_tensor(x, device=cuda)
    z, info = _solve(c, xt)
    zz = z.cpu().numpy()
    tol = TOL32 if x.dtype == np.float32 else TOL64
    assert _rel(zz, c["z"], x) <= tol, _rel(zz, c["z"], x)
    it_ref = c["iters"]
    slack = 0 if x.dtype == np.float64 else 4
    assert np.all(np.abs(info.image_iters - it_ref) <= slack), (info.image_iters, it_ref)
    assert info.converged == (int(c["status"]) == 0)
    # the certified gap: at most tol |x|^2 / 2 per converged image
    half = 0.5 * (x.astype(np.float64) ** 2).reshape(len(info.gaps), -1).sum(1)
    if info.converged:
        assert np.all(info.gaps <= float(c["tol"]) * half * (1 + 1e-9))
    d = info.dual.cpu().numpy()
    assert _rel(d, c["dual"], c["dual"]) <= 50 * tol


@pytest.mark.parametrize("name", ["iso2d_noise_f32", "iso2d_phantom_alpha_f32", "iso3d_f32"])
def test_host_arrays_staged_through_gpu(cuda, name):
    c = REF[name]
    z, info = _solve(c, c["x"].copy())
    assert isinstance(z, np.ndarray)
    assert _rel(z, c["z"], c["x"]) <= TOL32


def test_eight_by_256_noise_against_oracle(cuda):
    """8 x 256^2 N(0,1), gamma 0.1, tol 1e-6: z and iterations against the
    reference (C library when built, else the NumPy restatement)."""
    torch = _torch()
    from fastprox_b200 import TVIso, synth
    from oracle import ref_capi, tv_np
    x = synth.noise((8, 256, 256), 0)
    if ref_capi.available():
        r = ref_capi.solve(x, 0.1, tol=1e-6)
        zref, itref = r.z, r.iters
    else:
        zref, _, _, itref, _ = tv_np.tv_iso(x, 0.1, tol=1e-6)
    z, info = TVIso(2).solve(torch.as_tensor(x, device=cuda), 0.1, tol=1e-6)
    assert _rel(z.cpu().numpy(), zref, x) <= TOL32
    assert np.array_equal(info.image_iters, itref)


def test_bitwise_repeatable_and_batch_invariant(cuda):
    torch = _torch()
    from fastprox_b200 import TVIso, synth
    x = torch.as_tensor(synth.phantom(4, 64, 96, seed=21), device=cuda)
    op = TVIso(2)
    z1, i1 = op.solve(x, 0.2, tol=1e-7, max_iter=3000)
    z2, i2 = op.solve(x, 0.2, tol=1e-7, max_iter=3000)
    assert torch.equal(z1, z2) and np.array_equal(i1.image_iters, i2.image_iters)
    for b in range(4):  # alone: the same bits as in the batch
        zb, ib = TVIso(2).solve(x[b:b + 1].clone(), 0.2, tol=1e-7, max_iter=3000)
        assert torch.equal(zb[0], z1[b]) and ib.image_iters[0] == i1.image_iters[b]


def test_nan_inf_and_zero_step(cuda):
    torch = _torch()
    from fastprox_b200 import FastproxError, TVIso, synth
    x = synth.phantom(3, 32, 32, seed=3)
    x[1, 4, 5] = np.nan
    xt = torch.as_tensor(x, device=cuda)
    z, info = TVIso(2).solve(xt, 0.1)
    zz = z.cpu().numpy()
    assert np.isnan(zz[1]).all() and np.isfinite(zz[[0, 2]]).all()
    assert np.isnan(info.gaps[1]) and info.image_iters[1] == 0 and info.converged
    x[1, 4, 5] = np.inf
    with pytest.raises(FastproxError):
        TVIso(2).solve(torch.as_tensor(x, device=cuda), 0.1)
    y = torch.as_tensor(synth.phantom(2, 16, 16, seed=4), device=cuda)
    z0, i0 = TVIso(2).solve(y, 0.0)
    assert torch.equal(z0, y) and i0.iters == 0


def test_max_iter_reports_not_converged(cuda):
    torch = _torch()
    c = REF["iso_maxiter_f32"]
    z, info = _solve(c, torch.as_tensor(c["x"], device=cuda))
    assert not info.converged and np.all(info.image_iters == 37)
    assert _rel(z.cpu().numpy(), c["z"], c["x"]) <= TOL32


def test_strided_input_and_output(cuda):
    torch = _torch()
    from fastprox_b200 import TVIso, synth
    base = torch.as_tensor(synth.phantom(2, 40, 80, seed=5), device=cuda)
    view = base[:, :, ::2]
    out = torch.empty(2, 40, 80, device=cuda)[:, :, ::2]
    op = TVIso(2)
    z1, _ = op.solve(view, 0.3, tol=1e-7, max_iter=4000, out=out)
    z2, _ = TVIso(2).solve(view.contiguous(), 0.3, tol=1e-7, max_iter=4000)
    assert torch.equal(z1, z2)


def test_warm_start_from_converged_dual_takes_no_iterations(cuda):
    torch = _torch()
    from fastprox_b200 import TVIso, synth
    x = torch.as_tensor(synth.phantom(2, 48, 48, seed=6), device=cuda)
    op = TVIso(2)
    z, info = op.solve(x, 0.1, tol=1e-6)
    z2, info2 = op.solve(x, 0.1, tol=1e-6, dual=info.dual)
    assert info2.iters == 0
    assert torch.allclose(z2, z, atol=1e-5)
    # a warm start at a tighter tolerance continues from there
    z3, info3 = op.solve(x, 0.1, tol=1e-9, max_iter=20000, warm=True)
    assert info3.converged and info3.iters > 0


def test_conjugate_is_x_minus_prox(cuda):
    torch = _torch()
    from fastprox_b200 import TVIso, capi, synth
    import ctypes as C
    x = torch.as_tensor(synth.phantom(2, 32, 32, seed=7), device=cuda)
    op = TVIso(2)
    z, _ = op.solve(x, 1.0, tol=1e-8, max_iter=5000)
    out = torch.empty_like(x)
    L = capi.lib()
    ws = op.workspace(x)
    opt = capi.options(tol=1e-8, max_iter=5000)
    st = L.fp_prox_conj(op._op, 3.0, capi.ArrayRef(x).ref(), capi.ArrayRef(out).ref(), C.byref(opt), ws, None)
    assert st == capi.FP_OK
    torch.cuda.synchronize()
    assert torch.allclose(out, x - z, atol=1e-6)


def test_steps_per_image_on_device(cuda):
    torch = _torch()
    c = REF["iso_steps_f32"]
    z, info = _solve(c, torch.as_tensor(c["x"], device=cuda))
    assert _rel(z.cpu().numpy(), c["z"], c["x"]) <= TOL32
    assert info.image_iters[0] == 0
