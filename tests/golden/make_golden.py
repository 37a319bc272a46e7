"""Regenerates the golden fixtures of this directory. Runs only where the
reference is present (it reads its fixture file and runs the reference C
library built by ``oracle/Makefile``); the fixtures it writes are committed
and are all the tests need.

    make -C oracle && python tests/golden/make_golden.py REFERENCE_DIR

(or with the reference's checkout in the environment variable
FASTPROX_REFERENCE).

* ``cvxpy_images.npz`` -- the reference's own CVXPY/Clarabel golden vectors for
  the image-TV operators (tests/fixtures/reference_images.npz in the
  reference: every ``tv_iso*`` and ``tv_aniso*`` problem), copied as data.
* ``ref_vectors.npz``  -- outputs of the reference C library (``fp_prox`` /
  ``fp_prox_steps`` through its C ABI) on seeded inputs: z, per-image
  iterations, gaps and certified errors (``fp_workspace_image_info``), and the
  dual, for the cases listed in CASES; the conjugate cases (``fp_prox_conj``
  at the listed sigma, no dual) and images scaled far outside [2^-64, 2^65),
  which the reference solves at a power-of-two rescale.
"""

from __future__ import annotations

import os
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from fastprox_b200 import synth  # noqa: E402
from oracle import ref_capi  # noqa: E402

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
    # fp_prox_conj: y - prox(y) for positively homogeneous TV, at any sigma > 0; y itself at sigma = 0
    "conj_iso_s05_f64": (True, 2, lambda: synth.phantom(2, 20, 24, seed=17, dtype=np.float64), ("conj", 0.5),
                         None, None, 1e-9, 20000),
    "conj_iso_s3_f32": (True, 2, lambda: synth.phantom(2, 20, 24, seed=18), ("conj", 3.0), None,
                        lambda: synth.pixel_weights((20, 24), 19), 1e-6, 20000),
    "conj_iso_s0_f64": (True, 2, lambda: synth.phantom(1, 12, 10, seed=20, dtype=np.float64), ("conj", 0.0), None,
                        None, 1e-9, 1000),
    "conj_aniso_s2_f64": (False, 2, lambda: synth.phantom(2, 18, 22, seed=21, dtype=np.float64), ("conj", 2.0),
                          None, None, 1e-9, 20000),
    # max |x| outside [2^-64, 2^65): solved at a power-of-two rescale (image_util.hpp:56-70)
    "rescale_iso_m80_f64": (True, 2, lambda: synth.phantom(2, 24, 28, seed=22, dtype=np.float64) * 2.0 ** -80,
                            0.1 * 2.0 ** -80, None, None, 1e-9, 20000),
    "rescale_iso_p80_f64": (True, 2, lambda: synth.phantom(2, 24, 28, seed=23, dtype=np.float64) * 2.0 ** 80,
                            0.1 * 2.0 ** 80, None, lambda: synth.pixel_weights((24, 28), 24), 1e-9, 20000),
    "rescale_iso_m70_f32": (True, 2, lambda: (synth.phantom(2, 24, 28, seed=25) * np.float32(2.0 ** -70)),
                            0.1 * 2.0 ** -70, None, None, 1e-6, 20000),
    "rescale_aniso_m80_f64": (False, 2, lambda: synth.phantom(2, 24, 28, seed=26, dtype=np.float64) * 2.0 ** -80,
                              0.1 * 2.0 ** -80, None, None, 1e-9, 20000),
    "rescale_iso3d_p80_f64": (True, 3, lambda: synth.phantom3d(1, 6, 7, 8, seed=27, dtype=np.float64) * 2.0 ** 80,
                              0.2 * 2.0 ** 80, None, None, 1e-9, 20000),
}


def run_case(iso, k, x, gamma, w, sp, tol, max_iter):
    if isinstance(gamma, tuple) and gamma[0] == "conj":
        return ref_capi.solve(x, gamma[1], iso=iso, k=k, w=w, spatial=sp, tol=tol, max_iter=max_iter, conj=True)
    if isinstance(gamma, tuple):
        return ref_capi.solve(x, 0.0, iso=iso, k=k, w=w, spatial=sp, tol=tol, max_iter=max_iter,
                              steps=np.asarray(gamma[1]))
    return ref_capi.solve(x, gamma, iso=iso, k=k, w=w, spatial=sp, tol=tol, max_iter=max_iter)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FASTPROX_REFERENCE")
    if not ref:
        raise SystemExit("usage: make_golden.py REFERENCE_DIR (or FASTPROX_REFERENCE=REFERENCE_DIR)")
    # 1. the reference's CVXPY golden vectors for image TV, as data
    src = np.load(pathlib.Path(ref) / "tests" / "fixtures" / "reference_images.npz")
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
        conj = isinstance(gamma, tuple) and gamma[0] == "conj"
        # the reference leaves the per-image results of a conjugate at sigma = 0 unset
        unset = conj and gamma[1] == 0.0
        vec[f"{name}/gaps"] = np.zeros_like(r.gaps) if unset else r.gaps
        vec[f"{name}/zerrs"] = np.zeros_like(r.zerrs) if unset else r.zerrs
        if unset:
            vec[f"{name}/iters"] = np.zeros_like(r.iters)
        if r.dual is not None:
            vec[f"{name}/dual"] = r.dual.astype(x.dtype)
        vec[f"{name}/status"] = np.int32(r.status)
        vec[f"{name}/iso"] = np.int32(iso)
        vec[f"{name}/k"] = np.int32(k)
        vec[f"{name}/tol"] = np.float64(tol)
        vec[f"{name}/max_iter"] = np.int32(max_iter)
        if conj:
            vec[f"{name}/sigma"] = np.float64(gamma[1])
        elif isinstance(gamma, tuple):
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
