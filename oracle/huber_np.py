"""NumPy restatement of Huber-smoothed TV (test infrastructure only).

The reference plans this operator (ROADMAP.md, "Stage 1, Huber-smoothed TV":
``fp_op_tv_iso_huber``, ``fp_op_tv_aniso_huber``) but has no code for it, so
nothing of the reference pins these values: parity is unpinned. What pins
them here is the mathematics, checked in tests/test_oracle_huber.py: the
Tikhonov solution where no gradient passes delta (a linear solve), the TV
solution of the reference library as delta -> 0
(|z_delta - z_TV|^2 <= gamma delta sum alpha), and the gap certificate.

Problem, per image x (last k axes), with G = W D (forward differences,
w_a (z[p + e_a] - z[p]), zero at the last entry along a):
  isotropic:   min_z 1/2 |z - x|^2 + gamma sum_p alpha_p h(|(G z)_p|)
  anisotropic: min_z 1/2 |z - x|^2 + gamma sum_{a,p} beta_{a,p} h(|(G z)_{a,p}|)
h(t) = t^2 / (2 delta) for t <= delta, t - delta / 2 beyond (the reference's
Huber function, src/ops/pointwise.cpp:189-206). Dual: q with radii
r = gamma alpha (per pixel) or gamma beta (per component),
  max_q 1/2 |x|^2 - 1/2 |x - G^T q|^2 - sum delta |q|^2 / (2 r),  |q| <= r,
z = x - G^T q. Solved by dual FISTA with a constant momentum
(sqrt(kappa) - 1) / (sqrt(kappa) + 1), kappa = 1 + r_max L / delta, step
1 / L, L = 4 sum_a w_a^2 (the device's iteration, in double), stopped when the
gap (the sum of the Fenchel-Young gaps per pixel or component) is at most
tol |x|^2 / 2, checked every 4 iterations and at max_iter.
"""

from __future__ import annotations

import numpy as np


def _grad(z, w, k):
    """(k, ...) forward differences times the axis weights, zero at the last entry."""
    g = np.zeros((k,) + z.shape)
    for a in range(k):
        ax = z.ndim - k + a
        d = np.diff(z, axis=ax)
        sl = [slice(None)] * z.ndim
        sl[ax] = slice(0, z.shape[ax] - 1)
        g[a][tuple(sl)] = w[a] * d
    return g


def _div(q, w, k):
    """G^T q: sum_a w_a (q_a[p - e_a] - q_a[p]), q_a zero at the last entry."""
    out = np.zeros(q.shape[1:])
    for a in range(k):
        ax = q.ndim - 1 - k + a
        qa = q[a].copy()
        sl = [slice(None)] * qa.ndim
        sl[ax] = qa.shape[ax] - 1
        qa[tuple(sl)] = 0.0
        prev = np.zeros_like(qa)
        s_d = [slice(None)] * qa.ndim
        s_s = [slice(None)] * qa.ndim
        s_d[ax] = slice(1, None)
        s_s[ax] = slice(0, -1)
        prev[tuple(s_d)] = qa[tuple(s_s)]
        out += w[a] * (prev - qa)
    return out


def huber_h(t, delta):
    return np.where(t <= delta, t * t / (2.0 * delta), t - 0.5 * delta)


def gap(x, q, gamma, delta, w, k, iso, spatial=None):
    """The duality gap of (z = x - G^T q, q) and z."""
    z = x - _div(q, w, k)
    g = _grad(z, w, k)
    if iso:
        r = gamma * (np.ones(x.shape) if spatial is None else np.broadcast_to(spatial, x.shape))
        nrm = np.sqrt((g * g).sum(0))
        qq = (q * q).sum(0)
        pq = (g * q).sum(0)
        with np.errstate(divide="ignore", invalid="ignore"):
            t = np.where(r > 0, r * huber_h(nrm, delta) - pq + delta * qq / (2.0 * r), 0.0)
    else:
        r = gamma * (np.ones((k,) + x.shape) if spatial is None else np.broadcast_to(spatial, (k,) + x.shape))
        with np.errstate(divide="ignore", invalid="ignore"):
            t = np.where(r > 0, r * huber_h(np.abs(g), delta) - g * q + delta * q * q / (2.0 * r), 0.0)
    return float(t.sum()), z


def prox(x, gamma, delta, *, k=2, w=None, iso=True, spatial=None, tol=1e-12, max_iter=200000):
    """One image (the last k axes of x, float64): (z, q, gap, iters)."""
    x = np.asarray(x, np.float64)
    w = np.broadcast_to(np.asarray(1.0 if w is None else w, np.float64), (k,)).copy()
    wmax = float(w.max())
    if gamma == 0.0 or wmax == 0.0:
        return x.copy(), np.zeros((k,) + x.shape), 0.0, 0
    L = 4.0 * float((w * w).sum())
    tau = 1.0 / L
    if iso:
        r = gamma * (np.ones(x.shape) if spatial is None else np.broadcast_to(spatial, x.shape).astype(np.float64))
    else:
        r = gamma * (np.ones((k,) + x.shape) if spatial is None
                     else np.broadcast_to(spatial, (k,) + x.shape).astype(np.float64))
    rmax = float(r.max())
    kappa = 1.0 + rmax * L / delta
    beta = (np.sqrt(kappa) - 1.0) / (np.sqrt(kappa) + 1.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        shrink = np.where(r > 0, r / (r + tau * delta), 0.0)
    q = np.zeros((k,) + x.shape)
    v = q.copy()
    target = tol * 0.5 * float((x * x).sum())
    it = 0
    gp = np.inf
    while it < max_iter:
        z = x - _div(v, w, k)
        c = v + tau * _grad(z, w, k)
        if iso:
            c = c * shrink
            nrm = np.sqrt((c * c).sum(0))
            with np.errstate(divide="ignore", invalid="ignore"):
                sc = np.where(nrm > r, r / np.where(nrm > 0, nrm, 1.0), 1.0)
            qn = c * sc
        else:
            qn = np.clip(c * shrink, -r, r)
        v = qn + beta * (qn - q)
        q = qn
        it += 1
        if it % 4 == 0 or it == max_iter:
            gp, _ = gap(x, q, gamma, delta, w, k, iso, spatial)
            if gp <= target:
                break
    gp, z = gap(x, q, gamma, delta, w, k, iso, spatial)
    return z, q, gp, it
