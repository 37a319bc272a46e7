"""Regenerates the golden fixtures of this directory. Runs only where the
reference is present (it reads its fixture file and runs the reference C
library built by ``oracle/Makefile``); the fixtures it writes are committed
and are all the tests need.

    make -C oracle && python tests/golden/make_golden.py

* ``cvxpy_images.npz`` -- the reference's own CVXPY/Clarabel golden vectors for
  the image-TV operators (tests/fixtures/reference_images.npz in the
  reference: every ``tv_iso*`` and ``tv_aniso*`` problem), copied as data.
* ``ref_vectors.npz``  -- outputs of the reference C library (``fp_prox`` /
  ``fp_prox_steps`` through its C ABI) on seeded inputs: z, per-image
  iterations and gaps, and the dual, for the cases listed in CASES.
"""

from __future__ import annotations

import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fastprox_b200 import synth  # noqa: E402
from oracle import ref_capi  # noqa: E402

REF_FIXTURES = pathlib.Path("/root/reference/tests/fixtures/reference_images.npz")
OUT = pathlib.Path(__file__).resolve().parent

# name: (iso, k, x maker, gamma or steps, weights, spatial maker, tol, max_iter)
CASES = {
    "iso2d_noise_f32": (True, 2, lambda: synth.noise((2, 32, 32), 0), 0.1, None, None, 1e-6, 1000),
    "iso2d_noise_tight_f64": (True, 2, lambda: synth.noise((2, 24, 36), 1, np.float64), 0.3, [0.7, 1.3], None,
                              1e-10, 20000),
    "iso2d_phantom_alpha_f32": (True, 2, lambda: synth.phantom(2, 48, 40, seed=2), 0.1, None,
                                lambda: synth.pixel_weights((48, 40), 3), 1e-6, 2000),
    "iso2d_phantom_w_f32": (True, 2, lambda: synth.phantom(3, 40, 64, seed=4), 0.2, [1.0, 0.5], None, 1e-6, 3000),
    "iso2d_odd_f32": (True, 2, lambda: synth.phantom(2, 17, 23, seed=5), 0.15, None, None, 1e-7, 4000),
    "iso3d_f32": (True, 3, lambda: synth.phantom3d(2, 8, 10, 12, seed=6), 0.2, None, None, 1e-6, 3000),
    "iso3d_alpha_f64": (True, 3, lambda: synth.phantom3d(1, 6, 7, 8, seed=7, dtype=np.float64), 0.3, [1.0, 0.8, 1.2],
                        lambda: synth.pixel_weights((6, 7, 8), 8), 1e-8, 20000),
    "iso_steps_f32": (True, 2, lambda: synth.phantom(4, 32, 32, seed=9), ("steps", [0.0, 0.05, 0.1, 0.5]), None,
                      None, 1e-6, 3000),
    "iso_1d_f64": (True, 2, lambda: synth.noise((2, 1, 40), 10, np.float64), 0.5, None, None, 1e-9, 1000),
    "iso_maxiter_f32": (True, 2, lambda: synth.phantom(2, 32, 32, seed=11), 0.3, None, None, 1e-10, 37),
    "aniso2d_phantom_f32": (False, 2, lambda: synth.phantom(2, 32, 32, seed=12), 0.1, None, None, 1e-6, 1000),
    "aniso2d_noise_f64": (False, 2, lambda: synth.noise((2, 20, 28), 13, np.float64), 0.4, [1.2, 0.8], None, 1e-9,
                          5000),
    "aniso2d_edge_f32": (False, 2, lambda: synth.phantom(2, 24, 30, seed=14), 0.1, None,
                         lambda: synth.pixel_weights((2, 24, 30), 15), 1e-6, 1000),
    "aniso3d_f32": (False, 3, lambda: synth.phantom3d(2, 8, 10, 12, seed=16), 0.15, None, None, 1e-6, 2000),
}


def run_case(iso, k, x, gamma, w, sp, tol, max_iter):
    if isinstance(gamma, tuple):
        return ref_capi.solve(x, 0.0, iso=iso, k=k, w=w, spatial=sp, tol=tol, max_iter=max_iter,
                              steps=np.asarray(gamma[1]))
    return ref_capi.solve(x, gamma, iso=iso, k=k, w=w, spatial=sp, tol=tol, max_iter=max_iter)


def main():
    # 1. the reference's CVXPY golden vectors for image TV, as data
    src = np.load(REF_FIXTURES)
    keep = {}
    for key in src.files:
        case = str(src[key.split("/")[0] + "/case"])
        if case.startswith("tv_iso") or case.startswith("tv_aniso"):
            keep[key] = src[key]
    np.savez_compressed(OUT / "cvxpy_images.npz", **keep)
    # 2. reference C library outputs on seeded inputs
    vec = {}
    for name, (iso, k, mk, gamma, w, spk, tol, max_iter) in CASES.items():
        x = mk()
        sp = None if spk is None else spk()
        r = run_case(iso, k, x, gamma, w, sp, tol, max_iter)
        vec[f"{name}/x"] = x
        vec[f"{name}/z"] = r.z
        vec[f"{name}/iters"] = r.iters
        vec[f"{name}/gaps"] = r.gaps
        vec[f"{name}/dual"] = r.dual.astype(x.dtype)
        vec[f"{name}/status"] = np.int32(r.status)
        vec[f"{name}/iso"] = np.int32(iso)
        vec[f"{name}/k"] = np.int32(k)
        vec[f"{name}/tol"] = np.float64(tol)
        vec[f"{name}/max_iter"] = np.int32(max_iter)
        if isinstance(gamma, tuple):
            vec[f"{name}/steps"] = np.asarray(gamma[1], np.float64)
        else:
            vec[f"{name}/gamma"] = np.float64(gamma)
        if w is not None:
            vec[f"{name}/weights"] = np.asarray(w, np.float64)
        if sp is not None:
            vec[f"{name}/spatial"] = sp
        print(f"{name}: iters {r.iters.tolist()} status {r.status}")
    np.savez_compressed(OUT / "ref_vectors.npz", **vec)


if __name__ == "__main__":
    main()
