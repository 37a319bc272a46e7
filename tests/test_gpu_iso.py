"""Isotropic TV on the GPU against the reference (the parity tests proper).

Every call goes through the C ABI (libfastprox_b200.so) on CUDA tensors or
on host arrays staged through the GPU. The checks are the reference's own
outputs on the same seeded inputs (tests/golden/ref_vectors.npz), the
oracle at the 8 x 256^2 workload, the certificate, and the edge cases the
reference tests (NaN and Inf images, zero steps, single active axis,
max_iter, strided arrays, warm starts, conjugates).

Tolerances (the relative error |z - z_ref| / |z_ref|, 2-norms): 1e-5 in
float32 (FP32 iterates against the reference's FP64 ones) and 1e-9 in
float64; the largest entry error, relative to 1 + max|x| as in the
reference's fixture tests, within 5e-5 (float32) and 1e-8 (float64).
Iteration counts: equal in float64; in float32 within one gap-check period
or 20% (FP32 rounding of the iterates can shift a restart; on the 512^2
benchmark images the counts are equal). The dual is not unique (only
sum_a w_a D_a^T q_a is), so it is checked by its certificate: feasible, and
z = x - G^T q.
"""

import numpy as np
import pytest

from golden_data import ref_vectors

pytestmark = pytest.mark.gpu

REF = ref_vectors()
ISO = sorted(n for n, c in REF.items() if int(c["iso"]) == 1 and "sigma" not in c)
TOL32, TOL64 = 1e-5, 1e-9
MAX32, MAX64 = 5e-5, 1e-8


def _nrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


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


def _check_certificate(x, z, q, c, f32):
    """|q_p| <= gamma alpha_p and z = x - sum_a w_a D_a^T q_a (the reference's
    certificate, tests/python/test_tv_iso.py:22-58)."""
    k = int(c["k"])
    w = np.broadcast_to(np.asarray(c.get("weights", 1.0), np.float64), (k,))
    B = x.reshape((-1,) + x.shape[x.ndim - k:]).shape[0]
    gam = np.broadcast_to(np.asarray(c["steps"] if "steps" in c else c["gamma"], np.float64), (B,))
    img = x.shape[x.ndim - k:]
    xb = x.reshape((B,) + img).astype(np.float64)
    qb = q.reshape((k, B) + img)
    zb = z.reshape((B,) + img)
    al = c.get("spatial")
    eps = 1e-5 if f32 else 1e-12
    for b in range(B):
        r = gam[b] * (1.0 if al is None else al)
        nrm = np.sqrt((qb[:, b] ** 2).sum(0))
        assert np.all(nrm <= r * (1 + eps) + eps), (nrm - r).max()
        zz = xb[b].copy()
        for a in range(k):
            ua = qb[a, b]
            prev = np.zeros_like(ua)
            sl_d = [slice(None)] * k
            sl_s = [slice(None)] * k
            sl_d[a] = slice(1, None)
            sl_s[a] = slice(0, -1)
            prev[tuple(sl_d)] = ua[tuple(sl_s)]
            zz = zz + w[a] * (ua - prev)
        assert np.abs(zz - zb[b]).max() <= (2e-5 if f32 else 1e-10) * (1 + np.abs(xb[b]).max())


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
    f32 = x.dtype == np.float32
    assert _nrel(zz, c["z"]) <= (TOL32 if f32 else TOL64), _nrel(zz, c["z"])
    assert _rel(zz, c["z"], x) <= (MAX32 if f32 else MAX64), _rel(zz, c["z"], x)
    it_ref = c["iters"]
    slack = 0 if not f32 else np.maximum(4, 0.2 * it_ref)
    assert np.all(np.abs(info.image_iters - it_ref) <= slack), (info.image_iters, it_ref)
    assert info.converged == (int(c["status"]) == 0)
    # the certified gap: at most tol |x|^2 / 2 per converged image
    half = 0.5 * (x.astype(np.float64) ** 2).reshape(len(info.gaps), -1).sum(1)
    if info.converged:
        assert np.all(info.gaps <= float(c["tol"]) * half * (1 + 1e-9))
    d = info.dual.cpu().numpy().astype(np.float64)
    _check_certificate(x, zz, d, c, f32)


@pytest.mark.parametrize("name", ["iso2d_noise_f32", "iso2d_phantom_alpha_f32", "iso3d_f32"])
def test_host_arrays_staged_through_gpu(cuda, name):
    c = REF[name]
    z, info = _solve(c, c["x"].copy())
    assert isinstance(z, np.ndarray)
    assert _nrel(z, c["z"]) <= TOL32


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
    assert _nrel(z.cpu().numpy(), zref) <= TOL32
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
    assert _nrel(z.cpu().numpy(), c["z"]) <= TOL32


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
    # a warm start at a tighter tolerance continues from there (float32
    # iterates reach about 1e-8; float64 for tighter)
    z3, info3 = op.solve(x, 0.1, tol=1e-8, max_iter=20000, warm=True)
    assert info3.converged and info3.iters > 0
    x64 = x.double()
    op64 = TVIso(2)
    z4, i4 = op64.solve(x64, 0.1, tol=1e-6)
    z5, i5 = op64.solve(x64, 0.1, tol=1e-11, max_iter=50000, warm=True)
    assert i5.converged and 0 < i5.iters


def test_conjugate_is_x_minus_prox(cuda):
    torch = _torch()
    from fastprox_b200 import TVIso, capi, synth
    import ctypes as C
    x = torch.as_tensor(synth.phantom(2, 32, 32, seed=7), device=cuda)
    op = TVIso(2)
    z, _ = op.solve(x, 1.0, tol=1e-6, max_iter=3000)
    out = torch.empty_like(x)
    L = capi.lib()
    ws = op.workspace(x)
    opt = capi.options(tol=1e-6, max_iter=3000)
    st = L.fp_prox_conj(op._op, 3.0, capi.ArrayRef(x).ref(), capi.ArrayRef(out).ref(), C.byref(opt), ws, None)
    assert st in (capi.FP_OK, capi.FP_ENOTCONV)  # the same solve as z's, at gamma = 1
    torch.cuda.synchronize()
    assert torch.allclose(out, x - z, atol=1e-6)


def test_steps_per_image_on_device(cuda):
    torch = _torch()
    c = REF["iso_steps_f32"]
    z, info = _solve(c, torch.as_tensor(c["x"], device=cuda))
    assert _nrel(z.cpu().numpy(), c["z"]) <= TOL32
    assert info.image_iters[0] == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_3d_multi_tile_against_reference(cuda, dtype):
    """A volume spanning several tiles of the slice-marching 3D step in every
    axis (two x tiles, nine y tiles, five chunks of slices), with pixel
    weights, against the reference library on the same input."""
    torch = _torch()
    from fastprox_b200 import TVIso, synth
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    x = synth.phantom3d(1, 40, 70, 50, seed=21).astype(dtype)
    al = synth.pixel_weights((40, 70, 50), seed=22)
    tol = 1e-6 if dtype == np.float32 else 1e-10
    r = ref_capi.solve(x, 0.08, iso=True, k=3, spatial=al, tol=tol, max_iter=100000)
    z, info = TVIso(3, pixel_weights=al).solve(torch.as_tensor(x, device=cuda), 0.08, tol=tol, max_iter=100000)
    zz = z.cpu().numpy()
    assert _nrel(zz, r.z) <= (TOL32 if dtype == np.float32 else TOL64), _nrel(zz, r.z)
    it = int(info.image_iters[0])
    itr = int(r.iters[0])
    assert abs(it - itr) <= (max(4, 0.2 * itr) if dtype == np.float32 else 0), (it, itr)
