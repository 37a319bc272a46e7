"""Structure queries of a kept point on the GPU (fp_workspace_regions,
fp_workspace_kinks, fp_workspace_set_branch, fp_workspace_states / units /
constraint, fp_op_struct_kind, fp_workspace_deriv_exact) against the
reference library's answers on the same inputs (float64, gap tol 1e-12, so
that both find the same regions); output arrays on the host and the device,
int32 and int64 labels, strided outputs."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _kept(x, gamma, iso, beta=None, tol=1e-12):
    import torch
    from fastprox_b200 import TVAniso, TVIso, capi
    op = TVIso(2) if iso else TVAniso(2, edge_weights=beta)
    xt = torch.as_tensor(x, device="cuda")
    ws = op.workspace(xt, keep=True)
    L = capi.lib()
    z = torch.empty_like(xt)
    opt = capi.options(tol=tol, max_iter=500000, keep=True)
    st = L.fp_prox(op._op, gamma, capi.ArrayRef(xt).ref(), capi.ArrayRef(z).ref(), C.byref(opt), ws, None)
    assert st in (capi.FP_OK, capi.FP_ENOTCONV)
    return op, ws


def _regions(ws, shape, dtype, device, B):
    import torch
    from fastprox_b200 import capi
    td = {np.int32: torch.int32, np.int64: torch.int64}[dtype]
    lab = torch.full(shape, 7, dtype=td, device="cuda" if device else "cpu")
    sg = torch.zeros(shape, dtype=torch.int8, device="cuda" if device else "cpu")
    nreg = (C.c_int64 * B)()
    capi.check(capi.lib().fp_workspace_regions(ws, capi.ArrayRef(lab).ref(), capi.ArrayRef(sg).ref(), nreg, B),
               "regions")
    return lab.cpu().numpy().astype(np.int64), sg.cpu().numpy(), np.array(list(nreg))


@pytest.mark.parametrize("iso", [True, False], ids=["iso", "aniso"])
def test_regions_and_kinks_match_reference(cuda, iso):
    from fastprox_b200 import capi, synth
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    x = synth.phantom(2, 24, 30, seed=51).astype(np.float64)
    r = ref_capi.solve(x, 0.1, iso=iso, k=2, tol=1e-12, max_iter=500000, keep=True)
    lab_ref, nreg_ref = ref_capi.regions(r, 2)
    m_ref, c_ref = ref_capi.kinks(r, 1e-6)
    ex_ref, mu_ref = ref_capi.deriv_exact(r)
    ref_capi.release(r)
    op, ws = _kept(x, 0.1, iso)
    for dtype in (np.int32, np.int64):
        for device in (False, True):
            lab, sg, nreg = _regions(ws, x.shape, dtype, device, 2)
            assert np.array_equal(nreg, nreg_ref), (nreg, nreg_ref)
            assert np.array_equal(lab, lab_ref)
            assert np.all(sg == 1)
    import torch
    for device in (False, True):
        m = torch.full(x.shape, 5, dtype=torch.int8, device="cuda" if device else "cpu")
        c = C.c_int64()
        capi.check(capi.lib().fp_workspace_kinks(ws, 1e-6, capi.ArrayRef(m).ref(), C.byref(c)), "kinks")
        assert c.value == c_ref
        assert np.array_equal(m.cpu().numpy(), m_ref)
    ex, mu = C.c_int(), C.c_double()
    capi.check(capi.lib().fp_workspace_deriv_exact(ws, C.byref(ex), C.byref(mu)), "deriv_exact")
    assert ex.value == ex_ref
    assert abs(mu.value - mu_ref) <= 1e-6 * max(mu_ref, 1e-300), (mu.value, mu_ref)
    kind = C.c_int()
    capi.check(capi.lib().fp_op_struct_kind(op._op, C.byref(kind)), "kind")
    assert kind.value == (3 if iso else 1)


def test_states_units_constraint_and_strided_labels(cuda):
    import torch
    from fastprox_b200 import capi, synth
    L = capi.lib()
    x = synth.phantom(3, 16, 20, seed=52).astype(np.float64)
    x[1, 3, 4] = np.nan
    op, ws = _kept(x, 0.1, True, tol=1e-10)
    cnt, size = C.c_int64(), C.c_int64()
    capi.check(L.fp_workspace_units(ws, C.byref(cnt), C.byref(size)), "units")
    assert (cnt.value, size.value) == (3, 320)
    st = torch.full(x.shape, 9, dtype=torch.int8, device="cuda")
    nf = C.c_int64(-1)
    capi.check(L.fp_workspace_states(ws, capi.ArrayRef(st).ref(), C.byref(nf)), "states")
    assert nf.value == 0 and int(st.abs().sum()) == 0
    coef = torch.ones(x.shape, dtype=torch.float64)
    act = (C.c_int8 * 3)(1, 1, 1)
    capi.check(L.fp_workspace_constraint(ws, capi.ArrayRef(coef).ref(), act, 3), "constraint")
    assert float(coef.abs().sum()) == 0.0 and list(act) == [0, 0, 0]
    # labels into a strided (transposed) device view; the NaN image has none
    big = torch.full((3, 20, 16), 7, dtype=torch.int64, device="cuda")
    view = big.transpose(1, 2)
    nreg = (C.c_int64 * 3)()
    capi.check(L.fp_workspace_regions(ws, capi.ArrayRef(view).ref(), None, nreg, 3), "regions")
    lab = view.cpu().numpy()
    assert nreg[1] == -1 and np.all(lab[1] == -1)
    for b in (0, 2):
        assert lab[b].min() == 0 and lab[b].max() == nreg[b] - 1
        first = [np.argmax(lab[b].ravel() == c) for c in range(nreg[b])]
        assert first == sorted(first)  # numbered in order of first entries
    # wrong count, wrong dtype
    assert L.fp_workspace_regions(ws, None, None, nreg, 2) == capi.FP_ESHAPE
    bad = torch.zeros(x.shape, dtype=torch.float32)
    assert L.fp_workspace_states(ws, capi.ArrayRef(bad).ref(), None) == capi.FP_EDTYPE


def test_branch_override_matches_reference(cuda):
    """With a tolerance that makes every edge a kink, side -1 joins each image
    into one region (gx = the image mean of g) and +1 separates every entry
    (gx = g), as in the reference; NULL restores the default structure."""
    import torch
    from fastprox_b200 import capi, synth
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    L = capi.lib()
    x = synth.phantom(2, 18, 22, seed=53).astype(np.float64)
    g = np.random.default_rng(54).normal(size=x.shape)
    op, ws = _kept(x, 0.1, False)

    def vjp():
        gt = torch.as_tensor(g, device="cuda")
        gx = torch.empty_like(gt)
        gg = C.c_double()
        capi.check(L.fp_vjp(op._op, ws, capi.ArrayRef(gt).ref(), capi.ArrayRef(gx).ref(), C.byref(gg), None), "vjp")
        return gx.cpu().numpy(), gg.value

    gx0, gg0 = vjp()
    r = ref_capi.solve(x, 0.1, iso=False, k=2, tol=1e-12, max_iter=500000, keep=True)
    for side in (-1, 1):
        sd = np.full(x.shape, side, np.int8)
        capi.check(L.fp_workspace_set_branch(ws, capi.ArrayRef(torch.as_tensor(sd, device="cuda")).ref(), 1e3),
                   "branch")
        ref_capi.set_branch(r, sd, 1e3)
        gx, gg = vjp()
        gx_ref, gg_ref, _ = ref_capi.vjp(r, g, 2)
        assert np.abs(gx - gx_ref).max() <= 1e-12
        assert abs(gg - gg_ref) <= 1e-9 * (1 + abs(gg_ref))
        want = g.mean(axis=(1, 2), keepdims=True) if side < 0 else g
        assert np.abs(gx - want).max() <= 1e-12
    ref_capi.release(r)
    capi.check(L.fp_workspace_set_branch(ws, None, 0.0), "clear")
    gx, gg = vjp()
    assert np.array_equal(gx, gx0) and gg == gg0
    bad = np.full(x.shape, 2, np.int8)
    assert L.fp_workspace_set_branch(ws, capi.ArrayRef(bad).ref(), 1e-3) == capi.FP_EPARAM
    opi, wsi = _kept(x, 0.1, True, tol=1e-8)
    assert L.fp_workspace_set_branch(wsi, capi.ArrayRef(np.zeros(x.shape, np.int8)).ref(), 1e-3) == capi.FP_EINVAL


@pytest.mark.parametrize("iso", [True, False], ids=["iso", "aniso"])
def test_refine_reaches_the_tight_point(cuda, iso):
    """fp_workspace_refine from a loose kept call (gap tol 1e-4) to 1e-11
    gives the tight solve's z, and then the tight solve's derivative (both
    derivatives solved to 1e-12)."""
    import torch
    from fastprox_b200 import capi, synth
    L = capi.lib()
    x = synth.phantom(2, 20, 26, seed=55).astype(np.float64)
    g = torch.as_tensor(np.random.default_rng(56).normal(size=x.shape), device="cuda")

    def vjp(op, ws):
        capi.check(L.fp_workspace_set_deriv_tol(ws, 1e-12, 100000), "deriv_tol")
        gx = torch.empty_like(g)
        gg = C.c_double()
        capi.check(L.fp_vjp(op._op, ws, capi.ArrayRef(g).ref(), capi.ArrayRef(gx).ref(), C.byref(gg), None), "vjp")
        return gx.cpu().numpy(), gg.value

    op_t, ws_t = _kept(x, 0.1, iso, tol=1e-11)
    zt = torch.empty(x.shape, dtype=torch.float64, device="cuda")
    opt = capi.options(tol=1e-11, max_iter=500000, keep=True)
    capi.check(L.fp_prox(op_t._op, 0.1, capi.ArrayRef(torch.as_tensor(x, device="cuda")).ref(),
                         capi.ArrayRef(zt).ref(), C.byref(opt), ws_t, None), "tight", (capi.FP_OK,))
    gx_t, gg_t = vjp(op_t, ws_t)
    op, ws = _kept(x, 0.1, iso, tol=1e-4)
    zr = torch.empty_like(zt)
    info = capi.FpInfo()
    st = L.fp_workspace_refine(op._op, ws, 1e-11, 500000, capi.ArrayRef(zr).ref(), C.byref(info))
    assert st == capi.FP_OK
    rel = float((zr - zt).norm() / zt.norm())
    assert rel <= 1e-8, rel
    gx, gg = vjp(op, ws)
    assert np.linalg.norm(gx - gx_t) <= 1e-7 * np.linalg.norm(gx_t)
    assert abs(gg - gg_t) <= 1e-7 * (1 + abs(gg_t))
    assert L.fp_workspace_refine(op._op, ws, -1.0, 10, None, None) == capi.FP_EPARAM
