"""The PyTorch wrapper (fastprox_b200.torch.tv_iso / tv_aniso), the mirror of
the reference's fastprox.torch, tested as the reference tests its device path
(tests/python/test_device_tv.py:345-502): one step per image (each image's
result and gradients are a call's with its own step; a (B, 1) step broadcasts
over channels), pixel and edge weights against the reference C library's
solution and gradients (fp_vjp with keep_structure), one weight map per image,
differentiable axis weights, gradcheck in reverse and forward mode, warm
starts, ztol, and the argument errors. Float64 on the GPU."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SKEY = {True: "pixel_weights", False: "edge_weights"}


def _images(shape, seed):
    return np.random.default_rng(seed).normal(size=shape)


def _tv(iso):
    from fastprox_b200 import torch as fpt
    return fpt.tv_iso if iso else fpt.tv_aniso


def _spatial_weights(iso, img, seed, zeros=True):
    rng = np.random.default_rng(seed)
    size = img if iso else (len(img), *img)
    v = rng.uniform(0.3, 1.6, size)
    if zeros:
        v[rng.random(size) < 0.1] = 0.0
    return v


def _t(a, grad=False):
    import torch
    return torch.tensor(np.asarray(a, np.float64), device="cuda", requires_grad=grad)


@pytest.mark.parametrize("iso", [True, False])
def test_gamma_per_image(cuda, iso):
    x = _images((2, 3, 10, 11), 12)
    g = np.array([[0.15], [0.4]])
    c = np.random.default_rng(13).normal(size=x.shape)
    tv = _tv(iso)
    kw = dict(tol=1e-12, max_iter=10 ** 6)
    xt, gt = _t(x, True), _t(g, True)
    z = tv(xt, gt, **kw)
    z.backward(_t(c))
    z, gx, gg = z.detach().cpu().numpy(), xt.grad.cpu().numpy(), gt.grad.cpu().numpy()
    assert gg.shape == g.shape
    for b in range(2):
        xb = _t(x[b], True)
        gb = _t(float(g[b, 0]), True)
        zb = tv(xb, gb, **kw)
        zb.backward(_t(c[b]))
        zb, gxb, ggb = zb.detach().cpu().numpy(), xb.grad.cpu().numpy(), gb.grad.item()
        np.testing.assert_allclose(z[b], zb, atol=1e-10)
        np.testing.assert_allclose(gx[b], gxb, atol=1e-7 * (1 + np.abs(gxb).max()))
        assert float(gg[b, 0]) == pytest.approx(ggb, rel=1e-6, abs=1e-8)
    z0 = tv(_t(x), _t([[0.0], [0.4]]), **kw).detach().cpu().numpy()
    np.testing.assert_allclose(z0[0], x[0], atol=1e-12)
    np.testing.assert_allclose(z0[1], z[1], atol=1e-10)


@pytest.mark.parametrize("iso", [True, False])
def test_gamma_per_image_gradcheck(cuda, iso):
    import torch
    x = _images((2, 5, 6), 14)
    tv = _tv(iso)
    f = lambda x, g: tv(x, g, tol=1e-15, max_iter=10 ** 6)
    args = (_t(x, True), _t([0.3, 0.45], True))
    assert torch.autograd.gradcheck(f, args, check_forward_ad=True, atol=1e-5)


def _value_and_grads(iso, x, gamma, sw, c, ndim, **kw):
    tv = _tv(iso)
    xt, gt, st = _t(x, True), _t(gamma, True), _t(sw, True)
    z = tv(xt, gt, ndim=ndim, **{SKEY[iso]: st}, **kw)
    z.backward(_t(c))
    return z.detach().cpu().numpy(), xt.grad.cpu().numpy(), gt.grad.cpu().numpy(), st.grad.cpu().numpy()


@pytest.mark.parametrize("iso", [True, False])
@pytest.mark.parametrize("shape", [(2, 10, 12), (2, 5, 6, 7)])
def test_spatial_weights_match_reference(cuda, iso, shape):
    """Pixel or edge weights, some zero: the solution and the gradients in x,
    gamma and every weight against the reference C library's fp_vjp."""
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    k = len(shape) - 1
    img = shape[1:]
    x = _images(shape, 20)
    sw = _spatial_weights(iso, img, 21)
    c = np.random.default_rng(22).normal(size=shape)
    r = ref_capi.solve(x, 0.4, iso=iso, k=k, spatial=sw, tol=1e-14, max_iter=10 ** 6, keep=True)
    nparams = k + sw.size
    gxc, ggc, gpc = ref_capi.vjp(r, c, nparams, deriv_tol=1e-12)
    zc = r.z
    ref_capi.release(r)
    z, gx, gg, gs = _value_and_grads(iso, x, 0.4, sw, c, k, tol=1e-14, max_iter=10 ** 6, deriv_tol=1e-12)
    scale = 1 + np.abs(gxc).max()
    np.testing.assert_allclose(z, zc, atol=1e-10)
    np.testing.assert_allclose(gx, gxc, atol=1e-8 * scale)
    np.testing.assert_allclose(gs.reshape(-1), gpc[k:], atol=1e-8 * scale)
    assert float(gg) == pytest.approx(ggc, rel=1e-7, abs=1e-8)


@pytest.mark.parametrize("iso", [True, False])
def test_spatial_weights_per_image(cuda, iso):
    """A weight map per image: each image matches a call with its own map,
    and one map of the image shape broadcasts over the batch with its
    gradient summed."""
    x = _images((2, 9, 10), 23)
    maps = np.stack([_spatial_weights(iso, (9, 10), s) for s in (24, 25)], axis=0 if iso else 1)
    c = np.random.default_rng(26).normal(size=x.shape)
    kw = dict(tol=1e-13, max_iter=10 ** 6, deriv_tol=1e-12)
    z, gx, _, gs = _value_and_grads(iso, x, 0.3, maps, c, 2, **kw)
    assert gs.shape == maps.shape
    for b in range(2):
        mb = maps[b] if iso else maps[:, b]
        zb, gxb, _, gsb = _value_and_grads(iso, x[b], 0.3, mb, c[b], 2, **kw)
        np.testing.assert_allclose(z[b], zb, atol=1e-10)
        np.testing.assert_allclose(gx[b], gxb, atol=1e-8 * (1 + np.abs(gxb).max()))
        np.testing.assert_allclose(gs[b] if iso else gs[:, b], gsb, atol=1e-8 * (1 + np.abs(gsb).max()))
    one = maps[0] if iso else maps[:, 0]
    _, _, _, g1 = _value_and_grads(iso, x, 0.3, one, c, 2, **kw)
    _, _, _, g2 = _value_and_grads(iso, x, 0.3, np.stack([one, one], axis=0 if iso else 1), c, 2, **kw)
    np.testing.assert_allclose(g1, g2.sum(0) if iso else g2.sum(1), atol=1e-8 * (1 + np.abs(g1).max()))


@pytest.mark.parametrize("iso", [True, False])
def test_spatial_weights_gradcheck(cuda, iso):
    import torch
    x = _images((2, 5, 6), 27)
    sw = _spatial_weights(iso, (5, 6), 28, zeros=False)
    tv = _tv(iso)
    f = lambda x, s: tv(x, 0.35, **{SKEY[iso]: s}, tol=1e-15, max_iter=10 ** 6)
    assert torch.autograd.gradcheck(f, (_t(x, True), _t(sw, True)), check_forward_ad=True, atol=1e-5)


@pytest.mark.parametrize("iso", [True, False])
def test_axis_weights_gradient(cuda, iso):
    """Differentiable axis weights: the gradient is the reference's fp_vjp
    parameter gradient in the axis weights; gradcheck in both modes."""
    import torch
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    x = _images((2, 8, 9), 29)
    c = np.random.default_rng(30).normal(size=x.shape)
    w = np.array([0.7, 1.3])
    r = ref_capi.solve(x, 0.3, iso=iso, k=2, w=w, tol=1e-14, max_iter=10 ** 6, keep=True)
    _, _, gpc = ref_capi.vjp(r, c, 2, deriv_tol=1e-12)
    ref_capi.release(r)
    wt = _t(w, True)
    z = _tv(iso)(_t(x), 0.3, weights=wt, tol=1e-14, max_iter=10 ** 6, deriv_tol=1e-12)
    z.backward(_t(c))
    np.testing.assert_allclose(wt.grad.cpu().numpy(), gpc, rtol=1e-7, atol=1e-8)
    f = lambda x, w: _tv(iso)(x, 0.3, weights=w, tol=1e-15, max_iter=10 ** 6)
    assert torch.autograd.gradcheck(f, (_t(x[:1, :5, :6], True), _t(w, True)), check_forward_ad=True, atol=1e-5)


@pytest.mark.parametrize("iso", [True, False])
def test_warm_start_ztol_and_info(cuda, iso):
    """warm_start takes an earlier call's dual (fewer iterations, the same
    solution); ztol asks for tol = ztol^2; return_info gives the dual as a
    tensor; an unconverged solve warns."""
    import torch
    from fastprox_b200.torch import ConvergenceWarning
    x = _t(_images((2, 12, 14), 31))
    tv = _tv(iso)
    z1, i1 = tv(x, 0.2, tol=1e-10, max_iter=10 ** 6, return_info=True)
    assert isinstance(i1.dual, torch.Tensor) and tuple(i1.dual.shape) == (2, 2, 12, 14)
    z2, i2 = tv(x, 0.2, tol=1e-10, max_iter=10 ** 6, warm_start=i1.dual, return_info=True)
    assert i2.iters <= max(1, i1.iters // 2)
    torch.testing.assert_close(z2, z1, atol=1e-7, rtol=0)
    z3, i3 = tv(x, 0.2, ztol=1e-5, max_iter=10 ** 6, return_info=True)
    half = 0.5 * (x.double() ** 2).reshape(2, -1).sum(1).cpu().numpy()
    assert np.all(i3.gaps <= 1e-10 * half * (1 + 1e-9))
    with pytest.raises(ValueError):
        tv(x, 0.2, tol=1e-6, ztol=1e-3)
    with pytest.warns(ConvergenceWarning):
        tv(x, 0.2, tol=1e-14, max_iter=2)


def test_argument_errors(cuda):
    from fastprox_b200 import torch as fpt
    x = _t(np.zeros((2, 4, 5)))
    with pytest.raises(ValueError):
        fpt.tv_iso(x, 0.5, pixel_weights=_t(np.ones((3, 5))))
    with pytest.raises(ValueError):
        fpt.tv_aniso(x, 0.5, edge_weights=_t(np.ones((4, 5))))
    with pytest.raises(ValueError):
        fpt.tv_aniso(x, 0.5, edge_weights=_t(np.ones((3, 4, 5))))
    with pytest.raises(ValueError):
        fpt.tv_iso(x, _t([0.1, -0.2]))
    with pytest.raises(ValueError):
        fpt.tv_iso(_t(np.full((1, 3, 3), np.inf)), 0.1)
