"""The oracle pinned (CPU): the NumPy restatement of the reference's
isotropic fdpg against the reference C library's outputs (committed golden
vectors) and against the reference's CVXPY/Clarabel golden vectors; the
reference C library (when built) against the same CVXPY vectors."""

import numpy as np
import pytest

from golden_data import cvxpy_problems, ref_vectors
from oracle import ref_capi, tv_np

REF = ref_vectors()
ISO_CASES = sorted(n for n, c in REF.items() if int(c["iso"]) == 1 and "sigma" not in c)


@pytest.mark.parametrize("name", ISO_CASES)
def test_restatement_matches_reference_vectors(name):
    c = REF[name]
    x = c["x"]
    k = int(c["k"])
    steps = c.get("steps")
    z, dual, gaps, iters, conv = tv_np.tv_iso(
        x, float(c.get("gamma", 0.0)), k=k, w=c.get("weights", 1.0), alpha=c.get("spatial"),
        tol=float(c["tol"]), max_iter=int(c["max_iter"]), steps=steps)
    assert np.array_equal(iters, c["iters"]), (iters, c["iters"])
    if x.dtype == np.float64:
        assert np.abs(z - c["z"]).max() <= 1e-12 * (1 + np.abs(x).max())
    else:  # both round the same FP64 iterate to float32
        assert np.abs(z.astype(np.float64) - c["z"]).max() <= 2 * np.finfo(np.float32).eps * (1 + np.abs(x).max())
    np.testing.assert_allclose(gaps, c["gaps"], rtol=1e-6, atol=1e-12)


def _cvx(case_prefix):
    return [p for p in cvxpy_problems() if str(p["case"]).startswith(case_prefix)]


@pytest.mark.parametrize("case", ["tv_iso_2d", "tv_iso_3d"])
def test_restatement_matches_cvxpy(case):
    worst = 0.0
    for p in _cvx(case)[::2]:  # half of them keeps the CPU suite short
        k = 3 if "3d" in case else 2
        x = p["x"]
        w = p["param"].get("weights", 1.0)
        al = p["param"].get("pixel_weights")
        z, *_ = tv_np.prox_image(x, float(p["gamma"]), w, al, tol=1e-12, max_iter=200000)
        worst = max(worst, np.abs(z - p["z"]).max() / (1 + np.abs(x).max()))
    assert worst < 1e-5


@pytest.mark.skipif(not ref_capi.available(), reason="reference C library not built (make -C oracle)")
@pytest.mark.parametrize("case", ["tv_iso_2d", "tv_iso_3d", "tv_iso_2d_pixel", "tv_iso_3d_pixel",
                                  "tv_aniso_2d", "tv_aniso_3d", "tv_aniso_2d_edge", "tv_aniso_3d_edge"])
def test_reference_library_matches_cvxpy(case):
    worst = 0.0
    for p in [q for q in cvxpy_problems() if str(q["case"]) == case]:
        iso = case.startswith("tv_iso")
        k = 3 if "3d" in case else 2
        sp = p["param"].get("pixel_weights" if iso else "edge_weights")
        r = ref_capi.solve(p["x"], float(p["gamma"]), iso=iso, k=k, w=p["param"].get("weights"), spatial=sp,
                           tol=1e-14, max_iter=3_000_000)
        worst = max(worst, np.abs(r.z - p["z"]).max() / (1 + np.abs(p["x"]).max()))
    assert worst < 1e-7


def test_condat_matches_reference_single_axis():
    c = REF["iso_1d_f64"]
    z, dual, *_ = tv_np.tv_iso(c["x"], float(c["gamma"]), k=2, tol=float(c["tol"]))
    assert np.abs(z - c["z"]).max() <= 1e-13
    assert np.abs(dual - c["dual"]).max() <= 1e-12


def test_condat_weighted_against_dual_certificate():
    # exactness of the weighted 1D solve: dual feasibility and zero gap
    rng = np.random.default_rng(0)
    for _ in range(20):
        n = int(rng.integers(2, 40))
        y = rng.normal(size=n)
        w = rng.uniform(0, 2, n - 1) * (rng.uniform(size=n - 1) > 0.1)
        lam = float(rng.uniform(0.05, 2))
        z = tv_np.tv1d(y, lam, w)
        u = np.cumsum(y - z)[:-1]  # u_e = sum_{i<=e} (y - z)
        assert abs(np.sum(y - z)) <= 1e-10
        assert np.all(np.abs(u) <= lam * w + 1e-10)
        gap = lam * np.sum(w * np.abs(np.diff(z))) + np.sum(u * np.diff(z))
        assert abs(gap) <= 1e-9
