"""The implicit-differentiation VJP of isotropic TV on the GPU (fp_vjp on a
keep_structure point), against the reference's fp_vjp on the same inputs and
against float64 central finite differences of the forward; through the torch
autograd wrapper too. Bit-repeatable (exact fixed-point region sums)."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _keep_solve(x, gamma, tol, alpha=None, max_iter=200000):
    import torch
    from fastprox_b200 import TVIso, capi
    op = TVIso(2, pixel_weights=alpha)
    xt = x if isinstance(x, torch.Tensor) else torch.as_tensor(x, device="cuda")
    ws = op.workspace(xt, keep=True)
    L = capi.lib()
    capi.check(L.fp_workspace_set_stream(ws, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "stream")
    z = torch.empty_like(xt)
    opt = capi.options(tol=tol, max_iter=max_iter, keep=True)
    st = L.fp_prox(op._op, gamma, capi.ArrayRef(xt).ref(), capi.ArrayRef(z).ref(), C.byref(opt), ws, None)
    assert st in (capi.FP_OK, capi.FP_ENOTCONV)
    return op, ws, z


def _vjp(op, ws, g):
    import torch
    from fastprox_b200 import capi
    L = capi.lib()
    gt = torch.as_tensor(g, device="cuda")
    gx = torch.empty_like(gt)
    gg = C.c_double()
    capi.check(L.fp_vjp(op._op, ws, capi.ArrayRef(gt).ref(), capi.ArrayRef(gx).ref(), C.byref(gg), None), "fp_vjp")
    return gx.cpu().numpy(), gg.value


def _nrel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("dtype,tol,bound", [(np.float64, 1e-12, 1e-6), (np.float32, 1e-6, 5e-2)])
def test_matches_reference_vjp(cuda, dtype, tol, bound):
    from fastprox_b200 import synth
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    x = synth.phantom(2, 24, 32, seed=3).astype(dtype)
    g = np.random.default_rng(4).normal(size=x.shape).astype(dtype)
    r = ref_capi.solve(x, 0.1, iso=True, tol=tol, max_iter=200000, keep=True)
    gx_ref, gg_ref, _ = ref_capi.vjp(r, g, 2)
    ref_capi.release(r)
    op, ws, z = _keep_solve(x, 0.1, tol)
    gx, gg = _vjp(op, ws, g)
    assert _nrel(gx, gx_ref) <= bound, _nrel(gx, gx_ref)
    assert abs(gg - gg_ref) <= bound * (1 + abs(gg_ref)), (gg, gg_ref)


def test_finite_differences_float64(cuda):
    import torch
    from fastprox_b200 import TVIso, synth
    x = synth.phantom(1, 20, 24, seed=5).astype(np.float64)
    rng = np.random.default_rng(6)
    g = rng.normal(size=x.shape)
    op, ws, z = _keep_solve(x, 0.15, 1e-14)
    gx, gg = _vjp(op, ws, g)
    h = 1e-6
    worst = 0.0
    for _ in range(8):
        d = rng.normal(size=x.shape)
        zp, _ = TVIso(2).solve(torch.as_tensor(x + h * d, device="cuda"), 0.15, tol=1e-15, max_iter=500000)
        zm, _ = TVIso(2).solve(torch.as_tensor(x - h * d, device="cuda"), 0.15, tol=1e-15, max_iter=500000)
        fd = float((g * (zp.cpu().numpy() - zm.cpu().numpy())).sum() / (2 * h))
        an = float((gx * d).sum())
        worst = max(worst, abs(fd - an) / max(1e-12, abs(an)))
    # gamma
    zp, _ = TVIso(2).solve(torch.as_tensor(x, device="cuda"), 0.15 + h, tol=1e-15, max_iter=500000)
    zm, _ = TVIso(2).solve(torch.as_tensor(x, device="cuda"), 0.15 - h, tol=1e-15, max_iter=500000)
    fdg = float((g * (zp.cpu().numpy() - zm.cpu().numpy())).sum() / (2 * h))
    assert worst <= 1e-4, worst
    assert abs(fdg - gg) <= 1e-4 * max(1.0, abs(fdg)), (fdg, gg)


def test_repeatable_and_autograd(cuda):
    import torch
    from fastprox_b200 import synth
    from fastprox_b200.torch import tv_iso
    x = synth.phantom(4, 48, 64, seed=7)
    g = np.random.default_rng(8).normal(size=x.shape).astype(np.float32)
    gamma = float(np.float32(0.1))  # the autograd path takes gamma in x's dtype
    op, ws, z = _keep_solve(x, gamma, 1e-6)
    a1, g1 = _vjp(op, ws, g)
    a2, g2 = _vjp(op, ws, g)
    assert np.array_equal(a1, a2) and g1 == g2
    xt = torch.as_tensor(x, device=cuda).requires_grad_(True)
    gam = torch.tensor(0.1, device=cuda, requires_grad=True)
    zt = tv_iso(xt, gam, tol=1e-6)
    (zt * torch.as_tensor(g, device=cuda)).sum().backward()
    assert np.array_equal(xt.grad.cpu().numpy(), a1)
    assert abs(float(gam.grad) - g1) <= 1e-6 * (1 + abs(g1))


def test_loss_gradient_against_reference_and_differences(cuda):
    """The differentiation workload's shape in small, (2, 3, 64, 64) phantoms +
    noise 0.1, gamma 0.1, loss = MSE to the clean phantom, through the torch
    wrapper: the float64 VJP in x and gamma against the reference's fp_vjp at
    the same kept point (tol 1e-12) and against float64 central differences on
    32 random directions (h = 1e-5, both sides at the same fixed iteration
    count, within 1e-4 of the larger of the derivative and a tenth of a random
    direction's typical derivative); the float32 gradient's error
    against the float64 one is stated (its flat regions come from an iterate
    certified to about 1e-3 relative at tol 1e-6)."""
    import torch
    from fastprox_b200 import synth
    from fastprox_b200.torch import tv_iso
    from fastprox_b200.workloads import vjp_checks
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    noisy, clean = synth.phantom(6, 64, 64, seed=11, sigma=0.1, clean=True)
    noisy, clean = noisy.reshape(2, 3, 64, 64), clean.reshape(2, 3, 64, 64)
    res = vjp_checks(noisy, clean, ndir=32)
    assert res["fd_max_rel_err"] <= 1e-4, res
    assert res["fd_gamma_rel_err"] <= 1e-4, res
    assert res["f32_vs_f64_gx_rel_err"] <= 0.2, res  # stated, see the docstring
    x = torch.as_tensor(noisy, device=cuda).double().requires_grad_(True)
    c = torch.as_tensor(clean, device=cuda).double()
    g = torch.tensor(0.1, device=cuda, dtype=torch.float64, requires_grad=True)
    z = tv_iso(x, g, tol=1e-12, max_iter=10 ** 6, deriv_tol=1e-12)
    ((z - c) ** 2).mean().backward()
    cot = (2.0 * (z.detach() - c) / z.numel()).reshape(6, 64, 64).cpu().numpy()
    r = ref_capi.solve(noisy.reshape(6, 64, 64).astype(np.float64), 0.1, iso=True, tol=1e-12, max_iter=10 ** 6,
                       keep=True)
    gxr, ggr, _ = ref_capi.vjp(r, cot, 2, deriv_tol=1e-12)
    ref_capi.release(r)
    assert _nrel(x.grad.reshape(6, 64, 64).cpu().numpy(), gxr) <= 1e-6
    assert abs(float(g.grad) - ggr) <= 1e-6 * (1 + abs(ggr))
