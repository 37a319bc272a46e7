"""Huber-smoothed TV on the GPU (fp_b200_op_tv_iso_huber / _aniso_huber)
against the NumPy restatement (oracle/huber_np.py; the reference plans this
operator but has no code for it, so the oracle is pinned by the mathematics
in tests/test_oracle_huber.py): isotropic and anisotropic, 2D and 3D, with
and without pixel or edge weights, float64 (1e-9 relative, the same iteration
counts) and float32 (1e-5); the gap certificate; a warm start from the dual;
the operator's parameters; the derivatives refused (not built)."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _nrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


CASES = [  # (iso, k, weighted, shape)
    (True, 2, False, (2, 24, 30)),
    (True, 2, True, (2, 20, 26)),
    (False, 2, False, (2, 24, 30)),
    (False, 2, True, (2, 20, 26)),
    (True, 3, False, (1, 8, 9, 10)),
    (False, 3, True, (1, 7, 8, 9)),
]


def _inputs(iso, k, weighted, shape, seed):
    from fastprox_b200 import synth
    x = (synth.phantom(shape[0], shape[1], shape[2], seed=seed, dtype=np.float64) if k == 2
         else synth.phantom3d(shape[0], *shape[1:], seed=seed, dtype=np.float64))
    sw = None
    if weighted:
        img = shape[1:]
        sw = synth.pixel_weights(img if iso else (k,) + img, seed=seed + 1)
    return x, sw


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_matches_oracle(cuda, case, dtype):
    import torch
    from fastprox_b200 import TVAnisoHuber, TVIsoHuber
    from oracle import huber_np
    iso, k, weighted, shape = CASES[case]
    x, sw = _inputs(iso, k, weighted, shape, 40 + case)
    gamma, delta = 0.15, 0.02
    f64 = dtype == np.float64
    tol = 1e-12 if f64 else 1e-6
    Op = TVIsoHuber if iso else TVAnisoHuber
    op = Op(k, None, sw, delta=delta)
    z, info = op.solve(torch.as_tensor(x.astype(dtype), device=cuda), gamma, tol=tol, max_iter=200000)
    zz = z.cpu().numpy()
    assert info.converged
    for b in range(shape[0]):
        zr, qr, gr, itr = huber_np.prox(x[b].astype(dtype).astype(np.float64), gamma, delta, k=k, iso=iso,
                                        spatial=sw, tol=tol, max_iter=200000)
        assert _nrel(zz[b], zr) <= (1e-9 if f64 else 1e-5), (b, _nrel(zz[b], zr))
        if f64:
            assert abs(int(info.image_iters[b]) - itr) <= 4, (info.image_iters[b], itr)
        # the certificate of the returned point, recomputed independently
        q = info.dual.cpu().numpy()[:, b].astype(np.float64)
        gp, zq = huber_np.gap(x[b].astype(dtype).astype(np.float64), q, gamma, delta, np.ones(k), k, iso, sw)
        half = 0.5 * float((x[b] ** 2).sum())
        assert gp <= tol * half * (1 + 1e-6) + (0 if f64 else 1e-5 * half)
        assert np.abs(zq - zz[b]).max() <= (1e-10 if f64 else 1e-5) * (1 + np.abs(x[b]).max())


def test_warm_start_parameters_and_refusals(cuda):
    import torch
    from fastprox_b200 import TVIsoHuber, capi, synth
    x = torch.as_tensor(synth.phantom(2, 32, 40, seed=60, dtype=np.float64), device=cuda)
    op = TVIsoHuber(2, delta=0.05)
    z, info = op.solve(x, 0.2, tol=1e-10, max_iter=100000)
    z2, info2 = op.solve(x, 0.2, tol=1e-10, max_iter=100000, dual=info.dual)
    assert info2.iters == 0 and torch.allclose(z2, z, atol=1e-9)
    L = capi.lib()
    assert L.fp_op_nparams(op._op) == 3 and L.fp_op_name(op._op) == b"tv_iso_huber"
    bad = C.c_void_p()
    assert L.fp_b200_op_tv_iso_huber(2, None, None, 0.0, C.byref(bad)) == capi.FP_EPARAM
    assert L.fp_b200_op_tv_aniso_huber(2, None, None, float("nan"), C.byref(bad)) == capi.FP_EPARAM
    ws = op.workspace(x, keep=True)
    out = torch.empty_like(x)
    opt = capi.options(tol=1e-8, max_iter=100000, keep=True)
    capi.check(L.fp_workspace_set_stream(ws, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "stream")
    st = L.fp_prox(op._op, 0.2, capi.ArrayRef(x).ref(), capi.ArrayRef(out).ref(), C.byref(opt), ws, None)
    assert st == capi.FP_OK
    gx = torch.empty_like(x)
    assert L.fp_vjp(op._op, ws, capi.ArrayRef(x).ref(), capi.ArrayRef(gx).ref(), None, None) == capi.FP_EINVAL
