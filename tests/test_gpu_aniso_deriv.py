"""Derivatives of anisotropic TV on the GPU (fp_vjp / fp_jvp at a
keep_structure point): against the reference's fp_vjp / fp_jvp on the same
inputs (2D, 2D with edge weights, 3D, a single active axis, a zero step), the
adjoint identity <g, J d> = <J^T g, d> in float32, central finite differences
of the forward in float64, and torch autograd through tv_aniso.

The derivative is the one of the solution's piecewise-constant structure
(components of flat edges, tv_aniso.cpp:1012-1180): it is exact once both
sides find the same structure, so the float64 comparison is tight (1e-6
relative, 2-norm, at gap tol 1e-12)."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# name, shape, axis weights, edge weights, step
CASES = [
    ("2d", (2, 16, 20), [1.0, 0.8], False, 0.1),
    ("2d_edge_weights", (2, 12, 14), [1.0, 1.0], True, 0.1),
    ("3d", (1, 6, 7, 8), [1.0, 0.7, 1.2], False, 0.1),
    ("one_axis", (2, 8, 10), [0.0, 1.0], False, 0.1),
    ("zero_step", (1, 9, 11), [1.0, 1.0], False, 0.0),
]
BOUND = 1e-6


def _nrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _inputs(shape, w, beta, seed, dtype=np.float64):
    from fastprox_b200 import synth
    k = len(w)
    x = synth.phantom(shape[0], shape[1], shape[2], seed=seed) if k == 2 else \
        synth.phantom3d(shape[0], *shape[1:], seed=seed)
    x = x.astype(dtype).reshape(shape)
    b = synth.pixel_weights((k,) + shape[-k:], seed=seed + 1) if beta else None
    return x, b


def _ours(x, gamma, w, b, tol):
    import torch
    from fastprox_b200 import TVAniso, capi
    op = TVAniso(len(w), weights=np.asarray(w, np.float64), edge_weights=b)
    xt = torch.as_tensor(x, device="cuda")
    ws = op.workspace(xt, keep=True)
    L = capi.lib()
    capi.check(L.fp_workspace_set_stream(ws, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "stream")
    z = torch.empty_like(xt)
    opt = capi.options(tol=tol, max_iter=500000, keep=True)
    st = L.fp_prox(op._op, gamma, capi.ArrayRef(xt).ref(), capi.ArrayRef(z).ref(), C.byref(opt), ws, None)
    assert st in (capi.FP_OK, capi.FP_ENOTCONV)
    return op, ws, z


def _vjp(op, ws, g, P, device=False):
    import torch
    from fastprox_b200 import capi
    gt = torch.as_tensor(g, device="cuda")
    gx = torch.empty_like(gt)
    gp = torch.zeros(P, dtype=torch.float64, device="cuda" if device else "cpu")
    gg = C.c_double()
    capi.check(capi.lib().fp_vjp(op._op, ws, capi.ArrayRef(gt).ref(), capi.ArrayRef(gx).ref(), C.byref(gg),
                                 capi.ArrayRef(gp).ref()), "fp_vjp")
    return gx.cpu().numpy(), gg.value, gp.cpu().numpy()


def _jvp(op, ws, dx, dgamma, dp, device=True):
    import torch
    from fastprox_b200 import capi
    dxt = torch.as_tensor(dx, device="cuda")
    dz = torch.empty_like(dxt)
    dpt = None if dp is None else torch.as_tensor(dp, device="cuda" if device else "cpu")
    capi.check(capi.lib().fp_jvp(op._op, ws, capi.ArrayRef(dxt).ref(), float(dgamma),
                                 None if dpt is None else capi.ArrayRef(dpt).ref(), capi.ArrayRef(dz).ref()),
               "fp_jvp")
    return dz.cpu().numpy()


def _close(a, b):
    if np.linalg.norm(b) == 0.0:
        return np.linalg.norm(a) <= 1e-12
    return _nrel(a, b) <= BOUND


@pytest.mark.parametrize("name,shape,w,beta,gamma", CASES, ids=[c[0] for c in CASES])
def test_vjp_and_jvp_match_reference(cuda, name, shape, w, beta, gamma):
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    x, b = _inputs(shape, w, beta, seed=3)
    k = len(w)
    P = k + (b.size if beta else 0)
    rng = np.random.default_rng(5)
    g = rng.normal(size=x.shape)
    dx = rng.normal(size=x.shape)
    dp = rng.normal(size=P)
    r = ref_capi.solve(x, gamma, iso=False, k=k, w=w, spatial=b, tol=1e-12, max_iter=500000, keep=True)
    gx_ref, gg_ref, gp_ref = ref_capi.vjp(r, g, P)
    dz_ref = [ref_capi.jvp(r, dx, 0.0, None), ref_capi.jvp(r, dx, 0.3, dp)]
    ref_capi.release(r)
    op, ws, z = _ours(x, gamma, w, b, 1e-12)
    for dev in (False, True):
        gx, gg, gp = _vjp(op, ws, g, P, device=dev)
        assert _close(gx, gx_ref), _nrel(gx, gx_ref)
        assert abs(gg - gg_ref) <= BOUND * (1 + abs(gg_ref)), (gg, gg_ref)
        assert _close(gp[:k], gp_ref[:k]), (gp[:k], gp_ref[:k])
        if beta:
            assert _close(gp[k:], gp_ref[k:]), _nrel(gp[k:], gp_ref[k:])
        assert _close(_jvp(op, ws, dx, 0.0, None, device=dev), dz_ref[0])
        assert _close(_jvp(op, ws, dx, 0.3, dp, device=dev), dz_ref[1])


def test_adjoint_identity_float32(cuda):
    """<g, J(dx, dgamma, dtheta)> = <J^T g, dx> + ggamma dgamma + <gtheta, dtheta>
    on 4 x 64^2 phantoms with edge weights (float32 data, float64 sums)."""
    from fastprox_b200 import synth
    x = synth.phantom(4, 64, 64, seed=11)
    b = synth.pixel_weights((2, 64, 64), seed=12)
    P = 2 + b.size
    rng = np.random.default_rng(13)
    g = rng.normal(size=x.shape).astype(np.float32)
    dx = rng.normal(size=x.shape).astype(np.float32)
    dp = rng.normal(size=P)
    op, ws, z = _ours(x, 0.1, [1.0, 0.8], b, 1e-6)
    gx, gg, gp = _vjp(op, ws, g, P)
    dz = _jvp(op, ws, dx, 0.5, dp)
    lhs = float((g.astype(np.float64) * dz).sum())
    rhs = float((gx.astype(np.float64) * dx).sum() + gg * 0.5 + gp @ dp)
    assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + abs(rhs)), (lhs, rhs)


def test_finite_differences_float64(cuda):
    """Within one piece of the structure the prox is affine in x and gamma:
    central differences of the forward (h = 1e-7) match the JVP."""
    import torch
    from fastprox_b200 import TVAniso, synth
    x = synth.phantom(1, 20, 24, seed=21).astype(np.float64)
    rng = np.random.default_rng(22)
    op, ws, z = _ours(x, 0.12, [1.0, 1.0], None, 1e-14)
    h = 1e-7
    for _ in range(4):
        d = rng.normal(size=x.shape)
        an = _jvp(op, ws, d, 0.0, None)
        zp, _ = TVAniso(2).solve(torch.as_tensor(x + h * d, device="cuda"), 0.12, tol=1e-15, max_iter=500000)
        zm, _ = TVAniso(2).solve(torch.as_tensor(x - h * d, device="cuda"), 0.12, tol=1e-15, max_iter=500000)
        fd = (zp.cpu().numpy() - zm.cpu().numpy()) / (2 * h)
        assert _nrel(an, fd) <= 1e-4, _nrel(an, fd)
    an = _jvp(op, ws, np.zeros_like(x), 1.0, None)
    zp, _ = TVAniso(2).solve(torch.as_tensor(x, device="cuda"), 0.12 + h, tol=1e-15, max_iter=500000)
    zm, _ = TVAniso(2).solve(torch.as_tensor(x, device="cuda"), 0.12 - h, tol=1e-15, max_iter=500000)
    assert _nrel(an, (zp.cpu().numpy() - zm.cpu().numpy()) / (2 * h)) <= 1e-4


def test_torch_autograd(cuda):
    import torch
    from fastprox_b200 import synth
    from fastprox_b200.torch import tv_aniso
    x = torch.as_tensor(synth.phantom(2, 32, 32, seed=31), device=cuda).double().requires_grad_(True)
    gamma = torch.tensor(0.1, dtype=torch.float64, device=cuda, requires_grad=True)
    z = tv_aniso(x, gamma, tol=1e-12, max_iter=100000)
    gz = torch.randn_like(z)
    (z * gz).sum().backward()
    op, ws, _ = _ours(x.detach().cpu().numpy(), 0.1, [1.0, 1.0], None, 1e-12)
    gx, gg, _ = _vjp(op, ws, gz.cpu().numpy(), 2)
    assert _nrel(x.grad.cpu().numpy(), gx) <= 1e-12
    assert abs(float(gamma.grad) - gg) <= 1e-10 * (1 + abs(gg))
