"""Anisotropic TV on the GPU against the reference (ADBPG / FDPG-3 with the
exact 1D steps and the polish, all on the device) through the C ABI.

Checks: the reference's own outputs on seeded inputs (tests/golden/
ref_vectors.npz), the reference's CVXPY/Clarabel golden vectors at a tight
tolerance, the 8 x 256^2 workload against the reference library, bitwise
repeatability, NaN / zero-step / single-axis images. Tolerances as for the
isotropic tests: |z - z_ref| / |z_ref| <= 1e-5 (float32), 1e-9 (float64).
"""

import numpy as np
import pytest

from golden_data import cvxpy_problems, ref_vectors

pytestmark = pytest.mark.gpu

REF = ref_vectors()
ANISO = sorted(n for n, c in REF.items() if int(c["iso"]) == 0 and "sigma" not in c)


def _nrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _solve(c, x, **kw):
    from fastprox_b200 import TVAniso
    op = TVAniso(int(c["k"]), c.get("weights"), c.get("spatial"))
    return op.solve(x, float(c["gamma"]), tol=float(c["tol"]), max_iter=int(c["max_iter"]), **kw)


@pytest.mark.parametrize("name", ANISO)
def test_matches_reference_vectors(cuda, name):
    import torch
    c = REF[name]
    x = c["x"]
    z, info = _solve(c, torch.as_tensor(x, device=cuda))
    zz = z.cpu().numpy()
    f32 = x.dtype == np.float32
    assert _nrel(zz, c["z"]) <= (1e-5 if f32 else 1e-9), _nrel(zz, c["z"])
    assert info.converged
    half = 0.5 * (x.astype(np.float64) ** 2).reshape(len(info.gaps), -1).sum(1)
    assert np.all(info.gaps <= float(c["tol"]) * half * (1 + 1e-9))
    slack = 0 if not f32 else np.maximum(2, 0.2 * c["iters"])
    assert np.all(np.abs(info.image_iters - c["iters"]) <= slack), (info.image_iters, c["iters"])


@pytest.mark.parametrize("case", ["tv_aniso_2d", "tv_aniso_3d", "tv_aniso_2d_edge", "tv_aniso_3d_edge"])
def test_matches_cvxpy(cuda, case):
    import torch
    from fastprox_b200 import TVAniso
    worst = 0.0
    for p in [q for q in cvxpy_problems() if str(q["case"]) == case]:
        k = 3 if "3d" in case else 2
        x = torch.as_tensor(p["x"], device=cuda)  # float64
        op = TVAniso(k, p["param"].get("weights"), p["param"].get("edge_weights"))
        z, info = op.solve(x, float(p["gamma"]), tol=1e-14, max_iter=200000)
        worst = max(worst, float(np.abs(z.cpu().numpy() - p["z"]).max() / (1 + np.abs(p["x"]).max())))
    assert worst < 1e-7


def test_eight_by_256_against_reference(cuda):
    import torch
    from fastprox_b200 import TVAniso, synth
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    x = synth.phantom(8, 256, 256, seed=3)
    for gamma in (0.05, 0.1, 0.2):
        r = ref_capi.solve(x, gamma, iso=False, tol=1e-6)
        z, info = TVAniso(2).solve(torch.as_tensor(x, device=cuda), gamma, tol=1e-6)
        assert _nrel(z.cpu().numpy(), r.z) <= 1e-5, (gamma, _nrel(z.cpu().numpy(), r.z))
        assert info.converged
        assert np.all(np.abs(info.image_iters - r.iters) <= np.maximum(2, 0.2 * r.iters)), (info.image_iters, r.iters)


def test_repeatable_nan_and_zero_step(cuda):
    import torch
    from fastprox_b200 import TVAniso, synth
    x = synth.phantom(3, 40, 56, seed=5)
    x[2, 3, 3] = np.nan
    xt = torch.as_tensor(x, device=cuda)
    op = TVAniso(2)
    z1, i1 = op.solve(xt, 0.2, tol=1e-7)
    z2, i2 = op.solve(xt, 0.2, tol=1e-7)
    assert torch.equal(torch.nan_to_num(z1, 7.0), torch.nan_to_num(z2, 7.0))
    assert np.isnan(z1[2].cpu().numpy()).all() and i1.image_iters[2] == 0
    z0, i0 = op.solve(xt[:2].contiguous(), 0.0)
    assert torch.equal(z0, xt[:2]) and i0.iters == 0


def test_single_active_axis_is_exact_1d_tv(cuda):
    import torch
    from fastprox_b200 import TVAniso
    from oracle import tv_np
    x = np.random.default_rng(0).normal(size=(2, 1, 50))
    z, info = TVAniso(2).solve(torch.as_tensor(x, device=cuda), 0.4)
    for b in range(2):
        ref = tv_np.tv1d(x[b, 0], 0.4)
        assert np.abs(z.cpu().numpy()[b, 0] - ref).max() <= 1e-12


def test_warm_start_from_converged_dual_takes_no_iterations(cuda):
    """The dual of a solve restarts it at its first check (iteration 0), in
    float32 and float64; a warm start at a tighter tolerance continues."""
    import torch
    from fastprox_b200 import TVAniso, synth
    for dt in (torch.float32, torch.float64):
        x = torch.as_tensor(synth.phantom(2, 40, 48, seed=41), device=cuda).to(dt)
        op = TVAniso(2)
        z, info = op.solve(x, 0.1, tol=1e-6, max_iter=5000)
        z2, info2 = op.solve(x, 0.1, tol=1e-6, max_iter=5000, dual=info.dual)
        assert info2.iters == 0 and info2.converged
        assert torch.allclose(z2, z, atol=1e-5)
        tight = 1e-8 if dt == torch.float32 else 1e-11
        z3, info3 = op.solve(x, 0.1, tol=tight, max_iter=20000, warm=True)
        assert info3.converged


@pytest.mark.parametrize("k,edge", [(2, False), (2, True), (3, False)])
def test_warm_start_matches_reference(cuda, k, edge):
    """A warm start of a nearby problem from the reference's dual of the
    first (the reference's warm-start path: feasible dual, first check, the
    warm pass for two axes), against the reference library doing the same, in
    float64: z to 1e-9 and the same iteration counts."""
    import torch
    from fastprox_b200 import TVAniso, synth
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    shape = (2, 24, 30) if k == 2 else (1, 8, 9, 10)
    x = (synth.phantom(shape[0], shape[1], shape[2], seed=42) if k == 2
         else synth.phantom3d(shape[0], *shape[1:], seed=42)).astype(np.float64).reshape(shape)
    x2 = x + 0.01 * np.random.default_rng(43).normal(size=x.shape)
    beta = synth.pixel_weights((k,) + shape[-k:], seed=44) if edge else None
    r1 = ref_capi.solve(x, 0.1, iso=False, k=k, spatial=beta, tol=1e-10, max_iter=100000)
    r2 = ref_capi.solve(x2, 0.1, iso=False, k=k, spatial=beta, tol=1e-10, max_iter=100000, warm_dual=r1.dual)
    op = TVAniso(k, edge_weights=beta)
    xt = torch.as_tensor(x2, device=cuda)
    z, info = op.solve(xt, 0.1, tol=1e-10, max_iter=100000, dual=torch.as_tensor(r1.dual, device=cuda))
    zz = z.cpu().numpy()
    assert np.linalg.norm(zz - r2.z) <= 1e-9 * np.linalg.norm(r2.z), np.linalg.norm(zz - r2.z) / np.linalg.norm(r2.z)
    assert np.array_equal(info.image_iters, r2.iters), (info.image_iters, r2.iters)
