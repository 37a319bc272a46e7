"""Parameter gradients (axis weights, then pixel weights) of fp_vjp and the
forward derivative fp_jvp of isotropic TV on the GPU, against the reference's
fp_vjp / fp_jvp on the same inputs; the adjoint identity
<g, J d> = <J^T g, d> at float32; the conjugate at sigma = 0 (J = I).

Tolerance: 1e-6 relative (2-norm) in float64 at gap tol 1e-12, as for the
VJP in x (both sides stop their conjugate gradients at the certified error of
z, at least 1e-10)."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# name, shape, axis weights, pixel weights
CASES = [
    ("2d_w_alpha", (2, 12, 14), [1.0, 0.7], True),
    ("2d_w", (1, 16, 12), [0.6, 1.2], False),
    ("one_axis", (2, 10, 12), [0.0, 1.3], False),  # one active axis: exact 1D TV per row
    ("3d_alpha", (1, 6, 7, 8), [1.0, 0.8, 1.1], True),
]
BOUND = 1e-6


def _nrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _inputs(shape, w, alpha, seed, dtype=np.float64):
    from fastprox_b200 import synth
    k = len(w)
    rng = np.random.default_rng(seed)
    if k == 2:
        x = synth.phantom(shape[0], shape[1], shape[2], seed=seed)
    else:
        x = synth.phantom3d(shape[0], *shape[1:], seed=seed)
    x = x.astype(dtype).reshape(shape)
    al = rng.uniform(0.5, 1.5, size=shape[-k:]) if alpha else None
    return x, al


def _ours(x, gamma, w, al, tol, keep=True):
    import torch
    from fastprox_b200 import TVIso, capi
    op = TVIso(len(w), weights=np.asarray(w, np.float64), pixel_weights=al)
    xt = torch.as_tensor(x, device="cuda")
    ws = op.workspace(xt, keep=True)
    L = capi.lib()
    capi.check(L.fp_workspace_set_stream(ws, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "stream")
    z = torch.empty_like(xt)
    opt = capi.options(tol=tol, max_iter=500000, keep=keep)
    st = L.fp_prox(op._op, gamma, capi.ArrayRef(xt).ref(), capi.ArrayRef(z).ref(), C.byref(opt), ws, None)
    assert st in (capi.FP_OK, capi.FP_ENOTCONV)
    return op, ws, z


def _vjp(op, ws, g, P, gp_device=False):
    import torch
    from fastprox_b200 import capi
    L = capi.lib()
    gt = torch.as_tensor(g, device="cuda")
    gx = torch.empty_like(gt)
    gp = torch.zeros(P, dtype=torch.float64, device="cuda" if gp_device else "cpu")
    gg = C.c_double()
    capi.check(L.fp_vjp(op._op, ws, capi.ArrayRef(gt).ref(), capi.ArrayRef(gx).ref(), C.byref(gg),
                        capi.ArrayRef(gp).ref()), "fp_vjp")
    return gx.cpu().numpy(), gg.value, gp.cpu().numpy()


def _jvp(op, ws, dx, dgamma, dp, device=True):
    import torch
    from fastprox_b200 import capi
    L = capi.lib()
    dxt = torch.as_tensor(dx, device="cuda")
    dz = torch.empty_like(dxt)
    dpt = None if dp is None else torch.as_tensor(dp, device="cuda" if device else "cpu")
    st = L.fp_jvp(op._op, ws, capi.ArrayRef(dxt).ref(), float(dgamma),
                  None if dpt is None else capi.ArrayRef(dpt).ref(), capi.ArrayRef(dz).ref())
    capi.check(st, "fp_jvp")
    return dz.cpu().numpy()


@pytest.mark.parametrize("name,shape,w,alpha", CASES, ids=[c[0] for c in CASES])
def test_parameter_gradients_match_reference(cuda, name, shape, w, alpha):
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    x, al = _inputs(shape, w, alpha, seed=7)
    k = len(w)
    P = k + (al.size if alpha else 0)
    g = np.random.default_rng(8).normal(size=x.shape)
    r = ref_capi.solve(x, 0.12, iso=True, k=k, w=w, spatial=al, tol=1e-12, max_iter=500000, keep=True)
    gx_ref, gg_ref, gp_ref = ref_capi.vjp(r, g, P)
    ref_capi.release(r)
    op, ws, z = _ours(x, 0.12, w, al, 1e-12)
    for dev in (False, True):
        gx, gg, gp = _vjp(op, ws, g, P, gp_device=dev)
        assert _nrel(gx, gx_ref) <= BOUND, _nrel(gx, gx_ref)
        assert abs(gg - gg_ref) <= BOUND * (1 + abs(gg_ref)), (gg, gg_ref)
        assert _nrel(gp[:k], gp_ref[:k]) <= BOUND, (gp[:k], gp_ref[:k])
        if alpha:
            assert _nrel(gp[k:], gp_ref[k:]) <= BOUND, _nrel(gp[k:], gp_ref[k:])


@pytest.mark.parametrize("name,shape,w,alpha", CASES, ids=[c[0] for c in CASES])
def test_jvp_matches_reference(cuda, name, shape, w, alpha):
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    x, al = _inputs(shape, w, alpha, seed=9)
    k = len(w)
    P = k + (al.size if alpha else 0)
    rng = np.random.default_rng(10)
    dx = rng.normal(size=x.shape)
    dp = rng.normal(size=P)
    r = ref_capi.solve(x, 0.12, iso=True, k=k, w=w, spatial=al, tol=1e-12, max_iter=500000, keep=True)
    cases = [(dx, 0.0, None), (np.zeros_like(dx), 0.7, None), (np.zeros_like(dx), 0.0, dp), (dx, -0.4, dp)]
    refs = [ref_capi.jvp(r, d, dg, p) for d, dg, p in cases]
    ref_capi.release(r)
    op, ws, z = _ours(x, 0.12, w, al, 1e-12)
    for (d, dg, p), ref in zip(cases, refs):
        for dev in (True, False):
            dz = _jvp(op, ws, d, dg, p, device=dev)
            if np.linalg.norm(ref) == 0.0:
                assert np.linalg.norm(dz) <= 1e-12
            else:
                assert _nrel(dz, ref) <= BOUND, (dg, p is None, _nrel(dz, ref))


def test_adjoint_identity_float32(cuda):
    """<g, J(dx, dgamma, dtheta)> = <J^T g, dx> + ggamma dgamma + <gtheta, dtheta>
    on the 8 x 64^2 pixel-weighted batch (float32 iterates, float64 sums). Both
    systems solved to 1e-9 (by default they stop at the certified error of z,
    about 1e-3 at gap tol 1e-6, and the identity holds to that)."""
    from fastprox_b200 import capi, synth
    x = synth.phantom(8, 64, 64, seed=11)
    al = synth.pixel_weights((64, 64), seed=12)
    w = [1.0, 0.8]
    P = 2 + al.size
    rng = np.random.default_rng(13)
    g = rng.normal(size=x.shape).astype(np.float32)
    dx = rng.normal(size=x.shape).astype(np.float32)
    dp = rng.normal(size=P)
    op, ws, z = _ours(x, 0.1, w, np.asarray(al, np.float64), 1e-6)
    capi.check(capi.lib().fp_workspace_set_deriv_tol(ws, 1e-9, 20000), "deriv_tol")
    gx, gg, gp = _vjp(op, ws, g, P)
    dz = _jvp(op, ws, dx, 0.5, dp)
    lhs = float((g.astype(np.float64) * dz).sum())
    rhs = float((gx.astype(np.float64) * dx).sum() + gg * 0.5 + gp @ dp)
    assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + abs(rhs)), (lhs, rhs)


def test_conjugate_at_sigma_zero_is_identity(cuda):
    import torch
    from fastprox_b200 import TVIso, capi
    L = capi.lib()
    x = torch.as_tensor(np.random.default_rng(14).normal(size=(2, 9, 11)), device="cuda")
    op = TVIso(2)
    ws = op.workspace(x, keep=True)
    capi.check(L.fp_workspace_set_stream(ws, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "stream")
    out = torch.zeros_like(x)
    opt = capi.options(tol=1e-8, keep=True)
    capi.check(L.fp_prox_conj(op._op, 0.0, capi.ArrayRef(x).ref(), capi.ArrayRef(out).ref(), C.byref(opt), ws,
                              None), "conj")
    assert torch.equal(out, x)
    g = torch.randn_like(x)
    gx = torch.empty_like(x)
    gg = C.c_double()
    gp = torch.ones(2, dtype=torch.float64)
    capi.check(L.fp_vjp(op._op, ws, capi.ArrayRef(g).ref(), capi.ArrayRef(gx).ref(), C.byref(gg),
                        capi.ArrayRef(gp).ref()), "vjp")
    assert torch.equal(gx, g) and np.isnan(gg.value) and float(gp.abs().sum()) == 0.0
    dz = torch.empty_like(x)
    capi.check(L.fp_jvp(op._op, ws, capi.ArrayRef(g).ref(), 0.0, None, capi.ArrayRef(dz).ref()), "jvp")
    assert torch.equal(dz, g)
    capi.check(L.fp_jvp(op._op, ws, capi.ArrayRef(g).ref(), 1.0, None, capi.ArrayRef(dz).ref()), "jvp")
    assert bool(torch.isnan(dz).all())


def test_jvp_rejects_bad_arguments(cuda):
    import torch
    from fastprox_b200 import TVIso, capi
    L = capi.lib()
    x = torch.as_tensor(np.random.default_rng(15).normal(size=(1, 8, 8)), device="cuda")
    op = TVIso(2)
    ws = op.workspace(x, keep=True)
    out = torch.empty_like(x)
    # no kept point yet
    assert L.fp_jvp(op._op, ws, capi.ArrayRef(x).ref(), 0.0, None, capi.ArrayRef(out).ref()) == capi.FP_EINVAL
    opt = capi.options(tol=1e-8, keep=True)
    capi.check(L.fp_prox(op._op, 0.1, capi.ArrayRef(x).ref(), capi.ArrayRef(out).ref(), C.byref(opt), ws, None),
               "prox")
    dz = torch.empty_like(x)
    assert L.fp_jvp(op._op, ws, capi.ArrayRef(x).ref(), float("nan"), None,
                    capi.ArrayRef(dz).ref()) == capi.FP_EPARAM
    bad = torch.zeros(3, dtype=torch.float64)
    assert L.fp_jvp(op._op, ws, capi.ArrayRef(x).ref(), 0.0, capi.ArrayRef(bad).ref(),
                    capi.ArrayRef(dz).ref()) == capi.FP_ESHAPE
    assert L.fp_jvp(op._op, ws, capi.ArrayRef(x.float()).ref(), 0.0, None,
                    capi.ArrayRef(dz).ref()) == capi.FP_EDTYPE
    gp = torch.zeros(5, dtype=torch.float64)
    gg = C.c_double()
    assert L.fp_vjp(op._op, ws, capi.ArrayRef(x).ref(), capi.ArrayRef(dz).ref(), C.byref(gg),
                    capi.ArrayRef(gp).ref()) == capi.FP_ESHAPE
