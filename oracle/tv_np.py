"""NumPy FP64 restatement of the reference's isotropic image-TV prox (test
infrastructure; the checker, never the product).

Follows the reference step by step so that iterates and iteration counts can
be compared, not only the fixed point:

* ``prox_image``   -- ``TVIso::prox_img``           src/ops/tv_iso.cpp:333-415
* ``_fdpg``        -- ``TVIso::fdpg``               src/ops/tv_iso.cpp:424-543
* ``_divergence``  -- ``TVIso::divergence``         src/ops/tv_iso.cpp:251-270
* ``_grad``        -- ``TVIso::grad_rows``          src/ops/tv_iso.cpp:275-288
* ``_gap``         -- ``TVIso::gap``                src/ops/tv_iso.cpp:290-306
* ``rescale_exponent`` -- src/ops/image_util.hpp:56-65
* ``fista_t``      -- src/ops/image_util.hpp:72
* ``condat``       -- exact 1D TV by L. Condat's direct algorithm (IEEE SPL 20(11),
  2013) with per-edge radii, as the reference's src/ops/tv1d.cpp:84-236 uses it
  for a single active axis (tv_iso.cpp:381-398).

Element-wise arithmetic is done in the reference's order (no fused
multiply-add in NumPy), so iterates agree with the C library to rounding;
only the order of the long sums (mean, imbalance, |d|^2, gap, restart dot)
differs.
"""

from __future__ import annotations

import math

import numpy as np

K_CHECK = 4                     # tv_iso.cpp:106
K_MAX_SCALED_STEP = 2.0 ** 960  # core/op.hpp:48
DBL_MIN = np.finfo(np.float64).tiny


def fista_t(t: float) -> float:
    """image_util.hpp:72."""
    return 0.5 * (1.0 + math.sqrt(1.0 + 4.0 * t * t))


def _ilogb(v: float) -> int:
    return math.frexp(v)[1] - 1


def rescale_exponent(d: np.ndarray, gamma: float, step: float) -> int:
    """image_util.hpp:56-65: the power-of-two scale of an image far from 1."""
    m = float(np.max(np.abs(d))) if d.size else 0.0
    if not m > 0.0:
        return 0
    e = _ilogb(m)
    if -64 <= e <= 64:
        return 0
    top = max(gamma, step)
    if e < 0 and top > 0.0:
        e = min(0, max(e, _ilogb(top) + 1 - _ilogb(K_MAX_SCALED_STEP)))
    return e


def condat(y: np.ndarray, radius) -> np.ndarray:
    """Exact 1D TV prox of y with radius(e) on the edge (e, e + 1), by
    Condat's direct algorithm (the classic bound updates, no running sum).
    radius(len(y) - 1) may be anything: the end condition u_{n-1} = 0 is
    tested separately, as in src/ops/tv1d.cpp:200-229."""
    y = np.asarray(y, np.float64)
    n = len(y)
    z = np.empty(n)
    if n == 1:
        z[0] = y[0]
        return z
    k = k0 = km = kp = 0
    lk = radius(0)
    vmin, vmax = y[0] - lk, y[0] + lk
    umin, umax = lk, -lk

    def jump_down():
        nonlocal k, k0, km, kp, lk, vmin, vmax, umin, umax
        z[k0:km + 1] = vmin
        le = radius(km)
        k = k0 = kp = km = km + 1
        lk = radius(k)
        vmin, vmax = y[k] + (le - lk), y[k] + (le + lk)
        umin, umax = lk, -lk

    def jump_up():
        nonlocal k, k0, km, kp, lk, vmin, vmax, umin, umax
        z[k0:kp + 1] = vmax
        le = radius(kp)
        k = k0 = km = kp = kp + 1
        lk = radius(k)
        vmin, vmax = y[k] - (le + lk), y[k] - (le - lk)
        umin, umax = lk, -lk

    while True:
        while k < n - 1:
            yn = y[k + 1]
            ln = radius(k + 1)
            m = k - k0 + 2
            if yn + umin < vmin - ln:
                jump_down()
            elif yn + umax > vmax + ln:
                jump_up()
            else:
                k += 1
                umin += yn - vmin
                umax += yn - vmax
                if umin >= ln:
                    vmin += (umin - ln) / m
                    umin = ln
                    km = k
                if umax <= -ln:
                    vmax += (umax + ln) / m
                    umax = -ln
                    kp = k
        m = k - k0 + 1
        if umin < 0.0:
            jump_down()
        elif umax > 0.0:
            jump_up()
        else:
            z[k0:n] = vmin + umin / m
            return z


def tv1d(y: np.ndarray, lam, weights=None) -> np.ndarray:
    """prox of lam * sum_e w_e |z_{e+1} - z_e| for one 1D signal."""
    y = np.asarray(y, np.float64)
    n = len(y)
    if n < 2 or lam == 0.0:
        return y.copy()
    if weights is None:
        return condat(y, lambda e: lam)
    w = np.asarray(weights, np.float64)
    out = np.empty(n)
    s = 0
    for e in range(n):  # zero-weight edges split the signal into pieces
        if e == n - 1 or w[e] == 0.0:
            piece = y[s:e + 1]
            rad = np.append(lam * w[s:e], 0.0)
            out[s:e + 1] = condat(piece, lambda i: rad[i]) if len(piece) > 1 else piece
            s = e + 1
    return out


# ---------------------------------------------------------------------------
# Isotropic TV (tv_iso.cpp)
# ---------------------------------------------------------------------------


def _shift_prev(ua: np.ndarray, a: int) -> np.ndarray:
    """ua[p - e_a], 0 at the first entry along a."""
    out = np.zeros_like(ua)
    sl_dst = [slice(None)] * ua.ndim
    sl_src = [slice(None)] * ua.ndim
    sl_dst[a] = slice(1, None)
    sl_src[a] = slice(0, -1)
    out[tuple(sl_dst)] = ua[tuple(sl_src)]
    return out


def _divergence(d, u, wa):
    """z = d + sum_a wa_a (u_a[p] - u_a[p - e_a])  (tv_iso.cpp:251-270)."""
    z = d.copy()
    for a in range(d.ndim):
        if wa[a] == 0.0:
            continue
        z = z + wa[a] * (u[a] - _shift_prev(u[a], a))
    return z


def _grad(z, wa):
    """gv_a = wa_a (z[p + e_a] - z[p]), 0 past the end or for inactive axes
    (tv_iso.cpp:275-288)."""
    k = z.ndim
    g = np.zeros((k,) + z.shape)
    for a in range(k):
        if wa[a] == 0.0 or z.shape[a] < 2:
            continue
        dst = [slice(None)] * k
        hi = [slice(None)] * k
        lo = [slice(None)] * k
        dst[a] = slice(0, -1)
        hi[a] = slice(1, None)
        lo[a] = slice(0, -1)
        g[a][tuple(dst)] = wa[a] * (z[tuple(hi)] - z[tuple(lo)])
    return g


def _radius(gamma, alpha, bound):
    """tv_iso.cpp:180-185: gamma alpha_p capped at bound, 0 where alpha_p = 0."""
    if alpha is None:
        return gamma
    r = gamma * alpha
    r = np.where(r <= bound, r, bound)
    return np.where(alpha == 0.0, 0.0, r)


def _pnorm(g):
    nn = np.zeros(g.shape[1:])
    for a in range(g.shape[0]):
        nn = nn + g[a] * g[a]
    return np.sqrt(nn)


def _gap(z, u, wa, gamma, alpha, bound):
    """sum_p r_p |g_p| - <g_p, u_p>, g = W D z  (tv_iso.cpp:290-306)."""
    g = _grad(z, wa)
    dot = np.zeros(z.shape)
    for a in range(z.ndim):
        dot = dot + g[a] * u[a]
    return float(np.sum(_radius(gamma, alpha, bound) * _pnorm(g) - dot))


def _fdpg(d, wa_in, gamma_in, alpha, tol, max_iter, warm_dual, trace=None):
    """tv_iso.cpp:424-543 on one image (d already rescaled)."""
    k = d.ndim
    N = d.size
    wmax = max(wa_in)
    wa = [0.0] * k
    whmin = 1.0
    for a in range(k):
        if wa_in[a] != 0.0:
            wa[a] = wa_in[a] / wmax
            whmin = min(whmin, wa[a])
    mean = float(np.sum(d)) / N
    imbalance = float(np.sum(np.abs(d - mean)))
    gamma = gamma_in * wmax
    bound = 2.0 * imbalance / whmin + DBL_MIN
    if not gamma <= bound and alpha is None:
        gamma = bound
    L2 = sum(4.0 * w * w for w in wa)
    tau = 1.0 / L2
    if warm_dual is not None:
        u = np.array(warm_dual, np.float64) * wmax
    else:
        u = np.zeros((k,) + d.shape)
    # warm-start projection: inactive components and last entries zero, then the ball
    for a in range(k):
        last = [slice(None)] * k
        last[a] = slice(d.shape[a] - 1, d.shape[a])
        if wa[a] == 0.0:
            u[a] = 0.0
        else:
            u[a][tuple(last)] = 0.0
            u[a] = np.where(np.isfinite(u[a]), u[a], 0.0)
    nr = _pnorm(u)
    rp = _radius(gamma, alpha, bound) * np.ones(d.shape)
    sc = np.where(nr > rp, rp / np.where(nr > 0, nr, 1.0), 1.0)
    u = u * np.where(nr > rp, sc, 1.0)
    v = u.copy()
    target = tol * 0.5 * float(np.sum(d * d))

    def primal(uu):
        zz = _divergence(d, uu, wa)
        return zz, _gap(zz, uu, wa, gamma, alpha, bound)

    t = 1.0
    it = since = last = 0
    z = None
    gp = math.inf
    if warm_dual is not None:
        z, gp = primal(u)
    rad = _radius(gamma, alpha, bound)
    while not gp <= target and it < max_iter:
        zv = _divergence(d, v, wa)
        tn = fista_t(t)
        beta = (t - 1.0) / tn
        t = tn
        test = it % K_CHECK == 0
        gv = _grad(zv, wa)
        cv = np.zeros_like(u)
        for a in range(k):
            if wa[a] != 0.0:
                cv[a] = v[a] + tau * gv[a]
        nrm = _pnorm(cv)
        sc = np.where(nrm > rad, rad / np.where(nrm > 0, nrm, 1.0), 1.0)
        un = cv * sc
        up = float(np.sum((v - un) * (un - u))) if test else 0.0
        v = un + beta * (un - u)
        u = un
        since += 1
        restart = test and up > 0.0 and since >= last
        if restart:
            v = u.copy()
            t = 1.0
            last = since
            since = 0
        it += 1
        if trace is not None:
            trace.append((it, restart))
        if it % K_CHECK == 0 or it == max_iter:
            z, gp = primal(u)
    if not math.isfinite(gp):
        z, gp = primal(u)
    return z, u / wmax, max(gp, 0.0), it, gp <= target


def prox_image(x, gamma, w, alpha=None, tol=1e-6, max_iter=1000, warm_dual=None, trace=None):
    """TVIso::prox_img (tv_iso.cpp:333-415) on one image of k = x.ndim axes.

    Returns (z, dual (k, *shape), gap, iters, converged) in float64."""
    d = np.array(x, np.float64)
    k = d.ndim
    shape = d.shape
    if np.isinf(d).any():
        raise ValueError("Inf in image")
    if np.isnan(d).any():
        return (np.full(shape, np.nan), np.full((k,) + shape, np.nan), math.nan, 0, True)
    w = list(np.broadcast_to(np.asarray(w, np.float64), (k,)))
    wmax = max([w[a] for a in range(k) if shape[a] > 1], default=0.0)
    wa = [0.0] * k
    act = []
    for a in range(k):
        if gamma > 0.0 and w[a] > 0.0 and shape[a] > 1 and w[a] >= 1e-100 * wmax:
            wa[a] = w[a]
            act.append(a)
    alphamax = 1.0 if alpha is None else float(np.max(alpha))
    step_scale = max(w) * alphamax
    e = rescale_exponent(d, gamma, gamma * step_scale) if act else 0
    for a in range(k):
        if e and wa[a] > 0.0 and not math.ldexp(gamma * wa[a], -e) > 0.0:
            e = 0
    q = None if warm_dual is None else np.array(warm_dual, np.float64)
    g = gamma
    if e:
        d = np.ldexp(d, -e)
        if q is not None:
            q = np.ldexp(q, -e)
        g = math.ldexp(gamma, -e)
    gap, iters, conv = 0.0, 0, True
    if not act:
        z, dual = d.copy(), np.zeros((k,) + shape)
    elif len(act) == 1 and alpha is None:
        a = act[0]
        lam = g * w[a]
        z = np.apply_along_axis(lambda f: tv1d(f, lam), a, d)
        cs = np.cumsum(d - z, axis=a)
        dual = np.zeros((k,) + shape)
        qa = -cs / w[a]
        last = [slice(None)] * k
        last[a] = slice(shape[a] - 1, shape[a])
        qa[tuple(last)] = 0.0
        dual[a] = qa
    else:
        z, dual, gap, iters, conv = _fdpg(d, wa, g, alpha, tol, max_iter, q, trace)
    if e:
        z = np.ldexp(z, e)
        dual = np.ldexp(dual, e)
        gap = math.ldexp(gap, 2 * e)
    return z, dual, gap, iters, conv


def tv_iso(x, gamma, *, k=2, w=1.0, alpha=None, tol=1e-6, max_iter=1000, steps=None):
    """Batched over the leading axes of x (images the last k axes). Returns
    (z in x's dtype, dual (k, *x.shape), gaps, iters, converged per image)."""
    x = np.asarray(x)
    img = x.shape[x.ndim - k:]
    xb = x.reshape((-1,) + img)
    B = xb.shape[0]
    st = np.broadcast_to(np.asarray(gamma if steps is None else steps, np.float64).reshape(-1), (B,))
    z = np.empty(xb.shape, np.float64)
    dual = np.empty((k, B) + img)
    gaps, iters, conv = np.zeros(B), np.zeros(B, np.int64), np.zeros(B, bool)
    for b in range(B):
        zb, db, gaps[b], iters[b], conv[b] = prox_image(xb[b], float(st[b]), w, alpha, tol, max_iter)
        z[b] = zb
        dual[:, b] = db
    return (z.reshape(x.shape).astype(x.dtype), dual.reshape((k,) + x.shape), gaps, iters, conv)
