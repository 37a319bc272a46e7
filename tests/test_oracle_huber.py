"""The NumPy restatement of Huber-smoothed TV (oracle/huber_np.py), pinned by
the mathematics, since the reference has no code for this operator (its
ROADMAP.md plans it): the Tikhonov solution where every gradient stays below
delta (a linear solve), the reference library's TV solution as delta -> 0
(|z_delta - z_TV|^2 <= gamma delta sum alpha, the roadmap's gate), and the gap
certificate |z - z*|^2 <= 2 gap. CPU only."""

import numpy as np
import pytest

from oracle import huber_np, ref_capi


def _gmat(shape, w):
    """G as a (k n, n) matrix for a small image: column p is G e_p."""
    n = int(np.prod(shape))
    cols = []
    for p in range(n):
        e = np.zeros(n)
        e[p] = 1.0
        cols.append(huber_np._grad(e.reshape(shape), w, len(shape)).reshape(-1))
    return np.stack(cols, axis=1)


@pytest.mark.parametrize("iso", [True, False])
def test_quadratic_regime_is_tikhonov(iso):
    rng = np.random.default_rng(1)
    x = rng.normal(size=(5, 6)) * 0.01  # gradients far below delta
    gamma, delta, w = 0.7, 10.0, np.array([1.0, 0.6])
    G = _gmat(x.shape, w)
    # every |(G z)| <= delta: h(t) = t^2 / (2 delta), so z = (I + gamma / delta G^T G)^-1 x
    zt = np.linalg.solve(np.eye(x.size) + gamma / delta * G.T @ G, x.reshape(-1)).reshape(x.shape)
    z, q, gp, it = huber_np.prox(x, gamma, delta, k=2, w=w, iso=iso, tol=1e-20, max_iter=20000)
    assert np.abs(z - zt).max() <= 1e-12 * (1 + np.abs(x).max())


@pytest.mark.skipif(not ref_capi.available(), reason="reference library not built (make -C oracle)")
@pytest.mark.parametrize("iso", [True, False])
def test_small_delta_approaches_tv(iso):
    from fastprox_b200 import synth
    x = synth.phantom(1, 16, 20, seed=3, dtype=np.float64)[0]
    al = synth.pixel_weights((16, 20) if iso else (2, 16, 20), seed=4)
    gamma = 0.2
    r = ref_capi.solve(x[None], gamma, iso=iso, k=2, spatial=al, tol=1e-16, max_iter=10 ** 6)
    for delta in (1e-2, 1e-3, 1e-4):
        z, q, gp, it = huber_np.prox(x, gamma, delta, k=2, iso=iso, spatial=al, tol=1e-16, max_iter=10 ** 6)
        bound = gamma * delta * float(np.sum(al))
        assert float(((z - r.z[0]) ** 2).sum()) <= bound + 1e-12, (delta, float(((z - r.z[0]) ** 2).sum()), bound)


@pytest.mark.parametrize("iso,k", [(True, 2), (False, 2), (True, 3)])
def test_gap_certifies_the_error(iso, k):
    from fastprox_b200 import synth
    x = synth.phantom(1, 12, 14, seed=5, dtype=np.float64)[0] if k == 2 else \
        synth.phantom3d(1, 6, 7, 8, seed=5, dtype=np.float64)[0]
    zs, _, _, _ = huber_np.prox(x, 0.15, 0.02, k=k, iso=iso, tol=1e-22, max_iter=10 ** 6)
    z, q, gp, it = huber_np.prox(x, 0.15, 0.02, k=k, iso=iso, tol=1e-6, max_iter=10 ** 6)
    assert gp <= 1e-6 * 0.5 * float((x * x).sum())
    assert float(((z - zs) ** 2).sum()) <= 2 * gp + 1e-15
