"""Parity at the benchmarked sizes, and the rows the small golden cases leave
open, against the reference C library (the checker, oracle/_ref, built from the
reference's sources) through the C ABI on CUDA tensors:

* the 64 x 512^2 benchmark's own kind of images: isotropic TV with one
  pixel-weight map for the batch and gamma 0.05 / 0.1 / 0.2 (the quad launches
  of four iterations, their checks and the redo of a passing check), anisotropic
  TV with edge weights and the polish;
* rows wider than one 512-column block (the WIDE pair launch, halo columns);
* the error against the reference run in float64 to gap 1e-12, stated beside
  the certified error zerr, which must bound it;
* the per-image certified errors zerr, the conjugate fp_prox_conj at sigma 0,
  0.5, 2, 3, and images whose max |x| lies outside [2^-64, 2^65) (the
  reference's power-of-two rescale), against the reference's outputs
  (tests/golden/ref_vectors.npz).

Tolerances: |z - z_ref| / |z_ref| <= 1e-5 in float32, 1e-9 in float64; the
largest entry error relative to 1 + max|x| <= 5e-5 (float32); iteration
counts equal to the reference's on the benchmark images.
"""

import ctypes as C

import numpy as np
import pytest

from golden_data import ref_vectors

pytestmark = pytest.mark.gpu

REF = ref_vectors()
TOL32, TOL64, MAX32 = 1e-5, 1e-9, 5e-5


def _nrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _emax(a, b, x):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() / (1 + np.abs(x).max()))


def _ref():
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built (make -C oracle)")
    return ref_capi


def _per_image(a, b):
    return np.array([_nrel(a[i], b[i]) for i in range(len(a))])


def test_iso_benchmark_images_match_reference(cuda):
    """Three 512^2 phantoms of the benchmark's generator (one per gamma), the
    pixel-weight map U[0.5, 1.5], tol 1e-6: z, iteration counts, gaps and
    certified errors against the reference library on the same float32 input."""
    import torch
    from fastprox_b200 import TVIso, synth
    ref = _ref()
    x = synth.phantom(3, 512, 512, seed=0, sigma=0.1)
    al = synth.pixel_weights((512, 512), seed=1)
    steps = np.array([0.05, 0.1, 0.2])
    r = ref.solve(x, 0.0, iso=True, k=2, spatial=al, tol=1e-6, max_iter=20000, steps=steps)
    z, info = TVIso(2, pixel_weights=al).solve(torch.as_tensor(x, device=cuda), torch.as_tensor(steps, device=cuda),
                                               tol=1e-6, max_iter=20000)
    zz = z.cpu().numpy()
    rel = _per_image(zz, r.z)
    assert rel.max() <= TOL32, rel
    assert _emax(zz, r.z, x) <= MAX32
    assert np.array_equal(info.image_iters, r.iters), (info.image_iters, r.iters)
    assert info.converged
    half = 0.5 * (x.astype(np.float64) ** 2).reshape(3, -1).sum(1)
    assert np.all(info.gaps <= 1e-6 * half)
    # the certified errors follow the gaps (r = sqrt(2 gap) / |x|): within the
    # gaps' own agreement with the reference's float64 iterates
    np.testing.assert_allclose(info.zerr, r.zerrs, rtol=0.05)


def test_wide_rows_match_reference(cuda):
    """Rows of 1540 pixels: three 512-column blocks and a partial fourth per
    row band (the pair launch with halo columns), pixel weights."""
    import torch
    from fastprox_b200 import TVIso, synth
    ref = _ref()
    x = synth.phantom(2, 64, 1540, seed=31, sigma=0.1)
    al = synth.pixel_weights((64, 1540), seed=32)
    r = ref.solve(x, 0.1, iso=True, k=2, spatial=al, tol=1e-6, max_iter=20000)
    z, info = TVIso(2, pixel_weights=al).solve(torch.as_tensor(x, device=cuda), 0.1, tol=1e-6, max_iter=20000)
    zz = z.cpu().numpy()
    assert _per_image(zz, r.z).max() <= TOL32, _per_image(zz, r.z)
    assert _emax(zz, r.z, x) <= MAX32
    assert np.all(np.abs(info.image_iters - r.iters) <= 4), (info.image_iters, r.iters)


def test_error_against_float64_solution_at_gap_1e12(cuda):
    """One benchmark image (gamma 0.05, pixel weights): the float32 GPU result
    at tol 1e-6 against the reference in float64 at tol 1e-12 is within its
    certified error zerr (and about the reference's own float32-input error);
    the float64 GPU solve at tol 1e-12 matches that solution to 1e-9."""
    import torch
    from fastprox_b200 import TVIso, synth
    ref = _ref()
    x = synth.phantom(1, 512, 512, seed=0, sigma=0.1)
    al = synth.pixel_weights((512, 512), seed=1)
    r64 = ref.solve(x.astype(np.float64), 0.05, iso=True, k=2, spatial=al, tol=1e-12, max_iter=200000)
    r32 = ref.solve(x, 0.05, iso=True, k=2, spatial=al, tol=1e-6, max_iter=20000)
    op = TVIso(2, pixel_weights=al)
    z, info = op.solve(torch.as_tensor(x, device=cuda), 0.05, tol=1e-6, max_iter=20000)
    err = _nrel(z.cpu().numpy(), r64.z)
    err_ref = _nrel(r32.z, r64.z)
    assert err <= float(info.zerr[0]), (err, info.zerr)
    assert err <= 2 * err_ref + 1e-6, (err, err_ref)
    z64, i64 = TVIso(2, pixel_weights=al).solve(torch.as_tensor(x.astype(np.float64), device=cuda), 0.05,
                                               tol=1e-12, max_iter=200000)
    assert i64.converged
    assert _nrel(z64.cpu().numpy(), r64.z) <= TOL64, _nrel(z64.cpu().numpy(), r64.z)
    assert int(i64.image_iters[0]) == int(r64.iters[0])


def test_aniso_benchmark_images_match_reference(cuda):
    """Three 512^2 phantoms (one per gamma), edge weights (2, 512, 512)
    U[0.5, 1.5], tol 1e-6: the device ADBPG with exact 1D steps and the polish
    against the reference library."""
    import torch
    from fastprox_b200 import TVAniso, synth
    ref = _ref()
    x = synth.phantom(3, 512, 512, seed=0, sigma=0.1)
    beta = synth.pixel_weights((2, 512, 512), seed=1)
    steps = np.array([0.05, 0.1, 0.2])
    r = ref.solve(x, 0.0, iso=False, k=2, spatial=beta, tol=1e-6, max_iter=20000, steps=steps)
    z, info = TVAniso(2, edge_weights=beta).solve(torch.as_tensor(x, device=cuda),
                                                 torch.as_tensor(steps, device=cuda), tol=1e-6, max_iter=20000)
    zz = z.cpu().numpy()
    assert _per_image(zz, r.z).max() <= TOL32, _per_image(zz, r.z)
    assert _emax(zz, r.z, x) <= MAX32
    assert info.converged
    assert np.all(np.abs(info.image_iters - r.iters) <= np.maximum(2, 0.2 * r.iters)), (info.image_iters, r.iters)


@pytest.mark.parametrize("name", sorted(n for n, c in REF.items() if "sigma" not in c))
def test_certified_errors_match_reference(cuda, name):
    """zerr = r + round (u (1 + r) + a / |x|), r = sqrt(2 gap) / |x| per image
    (the reference's certified_error), against the reference's own values: to
    1e-6 in float64 (same iterates, same gaps), and within the float32
    iterates' gap agreement otherwise."""
    import torch
    from fastprox_b200 import TVAniso, TVIso
    c = REF[name]
    x = c["x"]
    k = int(c["k"])
    Op = TVIso if int(c["iso"]) else TVAniso
    op = Op(k, c.get("weights"), c.get("spatial"))
    gamma = torch.as_tensor(c["steps"], device=cuda) if "steps" in c else float(c["gamma"])
    _, info = op.solve(torch.as_tensor(x, device=cuda), gamma, tol=float(c["tol"]), max_iter=int(c["max_iter"]))
    zr = c["zerrs"]
    if x.dtype == np.float64:
        np.testing.assert_allclose(info.zerr, zr, rtol=1e-6, atol=1e-300)
    else:
        # float32 iterates resolve a gap to about 2e-8 |x|^2 (each pixel's term
        # rounded to float32 before its FP64 sum), i.e. r = sqrt(2 gap) / |x| to
        # about 2e-4: a polished anisotropic image whose gap is below that may
        # read 0 here and a rounding-level value in the reference's FP64 iterates
        np.testing.assert_allclose(info.zerr, zr, rtol=0.25, atol=2e-4)


@pytest.mark.parametrize("name", sorted(n for n, c in REF.items() if "sigma" in c))
def test_conjugate_matches_reference(cuda, name):
    """fp_prox_conj (y - prox(y) for positively homogeneous TV, y at sigma = 0)
    against the reference's fp_prox_conj on the same input."""
    import torch
    from fastprox_b200 import TVAniso, TVIso, capi
    c = REF[name]
    x = torch.as_tensor(c["x"], device=cuda)
    k = int(c["k"])
    Op = TVIso if int(c["iso"]) else TVAniso
    op = Op(k, c.get("weights"), c.get("spatial"))
    out = torch.empty_like(x)
    ws = op.workspace(x)
    L = capi.lib()
    capi.check(L.fp_workspace_set_stream(ws, C.c_void_p(torch.cuda.current_stream().cuda_stream)), "stream")
    opt = capi.options(tol=float(c["tol"]), max_iter=int(c["max_iter"]))
    info = capi.FpInfo()
    st = L.fp_prox_conj(op._op, float(c["sigma"]), capi.ArrayRef(x).ref(), capi.ArrayRef(out).ref(), C.byref(opt),
                        ws, C.byref(info))
    assert st == int(c["status"]), (st, int(c["status"]))
    torch.cuda.synchronize()
    zz = out.cpu().numpy()
    f32 = c["x"].dtype == np.float32
    assert _nrel(zz, c["z"]) <= (TOL32 if f32 else TOL64), _nrel(zz, c["z"])
    if float(c["sigma"]) == 0.0:
        assert np.array_equal(zz, c["x"])
        return
    B = len(c["iters"])
    gaps, its, zerr = np.zeros(B), np.zeros(B, np.int32), np.zeros(B)
    capi.check(L.fp_workspace_image_info(ws, gaps.ctypes.data_as(C.POINTER(C.c_double)),
                                         its.ctypes.data_as(C.POINTER(C.c_int)),
                                         zerr.ctypes.data_as(C.POINTER(C.c_double)), B), "image_info")
    if not f32:
        assert np.array_equal(its, c["iters"]), (its, c["iters"])
        # the prox behind the conjugate solves y / sigma: a gap below 1e-13 of
        # its |y / sigma|^2 / 2 is at the rounding of the FP64 sums (a polished
        # anisotropic point), and r = sqrt(2 gap) / |y / sigma| then below 5e-7
        half = 0.5 * ((c["x"].astype(np.float64) / float(c["sigma"])) ** 2).reshape(B, -1).sum(1)
        np.testing.assert_allclose(gaps, c["gaps"], rtol=1e-6, atol=1e-13 * half.min())
        np.testing.assert_allclose(zerr, c["zerrs"], rtol=1e-6, atol=5e-7)


@pytest.mark.parametrize("name", sorted(n for n in REF if n.startswith("rescale_")))
def test_rescaled_images_match_reference(cuda, name):
    """max |x| of 2^-80, 2^80 (float64) and 2^-70 (float32): the set-up's
    rescaling exponent, the scaled solve and the unscaled outputs (z, the
    dual, the gaps at the input's scale) against the reference."""
    import torch
    from fastprox_b200 import TVAniso, TVIso
    c = REF[name]
    x = c["x"]
    k = int(c["k"])
    Op = TVIso if int(c["iso"]) else TVAniso
    z, info = Op(k, c.get("weights"), c.get("spatial")).solve(torch.as_tensor(x, device=cuda), float(c["gamma"]),
                                                             tol=float(c["tol"]), max_iter=int(c["max_iter"]))
    zz = z.cpu().numpy()
    f32 = x.dtype == np.float32
    assert _nrel(zz, c["z"]) <= (TOL32 if f32 else TOL64), _nrel(zz, c["z"])
    assert info.converged
    if not f32:
        assert np.array_equal(info.image_iters, c["iters"]), (info.image_iters, c["iters"])
        np.testing.assert_allclose(info.gaps, c["gaps"], rtol=1e-6)
        d = info.dual.cpu().numpy()
        scale = np.abs(c["dual"]).max()
        assert np.abs(d - c["dual"]).max() <= 1e-7 * scale
