"""Ragged batches (fp_b200_batch_*): images of mixed sizes, steps and
tolerances in one set of launches, against the per-image solve (fp_prox) and
against the reference C library on the same images; the same bits for an
image alone and in a mix; continuous admission."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(64, 96), (96, 64), (128, 160), (40, 50), (33, 37), (1, 80), (200, 32)]


def _nrel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _images(cuda):
    import torch
    from fastprox_b200 import synth
    rng = np.random.default_rng(0)
    out = []
    for i, (h, w) in enumerate(SHAPES):
        x = torch.as_tensor(synth.phantom(1, h, w, seed=i)[0], device=cuda)
        out.append((x, float(rng.uniform(0.02, 0.3)), float(10 ** rng.uniform(-6, -4))))
    return out


def _run_all(b):
    res = {}
    while b.pending:
        for slot, z, gap, it, conv in b.run(steps=8):
            res[slot] = (z, gap, it, conv)
    return res


def test_matches_per_image_solves(cuda):
    from fastprox_b200 import TVIso
    from fastprox_b200.batch import RaggedBatch
    imgs = _images(cuda)
    b = RaggedBatch(max_images=16, max_pixels=200_000)
    slots = [b.admit(x, g, t, max_iter=5000) for x, g, t in imgs]
    res = _run_all(b)
    for (x, g, t), s in zip(imgs, slots):
        zr, info = TVIso(2).solve(x[None], g, tol=t, max_iter=5000)
        z, gap, it, conv = res[s]
        assert conv == info.converged
        assert _nrel(z, zr[0]) <= 1e-5, (x.shape, _nrel(z, zr[0]))
        assert abs(it - int(info.image_iters[0])) <= max(4, 0.2 * it), (x.shape, it, info.image_iters)


def test_matches_reference_library(cuda):
    """Each image of the mixed batch (its own step and tolerance, with quads
    and pairs where its rows allow) against the reference's fp_prox on the
    same float32 input: 1e-5 relative, the float32 parity tolerance."""
    from fastprox_b200.batch import RaggedBatch
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    imgs = _images(cuda)
    b = RaggedBatch(max_images=16, max_pixels=200_000)
    slots = [b.admit(x, g, t, max_iter=5000) for x, g, t in imgs]
    res = _run_all(b)
    for (x, g, t), s in zip(imgs, slots):
        r = ref_capi.solve(x.cpu().numpy()[None], g, iso=True, k=2, tol=t, max_iter=5000)
        z = res[s][0].double().cpu().numpy()
        err = float(np.linalg.norm(z - r.z[0]) / max(np.linalg.norm(r.z[0]), 1e-300))
        assert err <= 1e-5, (x.shape, err)


def test_alone_equals_in_the_mix_and_continuous_admission(cuda):
    import torch
    from fastprox_b200.batch import RaggedBatch
    imgs = _images(cuda)
    alone = []
    for x, g, t in imgs:
        b = RaggedBatch(max_images=2, max_pixels=100_000)
        s = b.admit(x, g, t, max_iter=5000)
        alone.append(_run_all(b)[s])
    # the mix, admitted in two waves while the first iterates; a finished
    # image's slot is reused, so results are kept per request
    b = RaggedBatch(max_images=16, max_pixels=200_000)
    owner, res = {}, {}
    for k in range(4):
        owner[b.admit(*imgs[k], max_iter=5000)] = k
    for slot, z, gap, it, conv in b.run(steps=4):
        res[owner.pop(slot)] = (z, gap, it, conv)
    for k in range(4, len(imgs)):
        owner[b.admit(*imgs[k], max_iter=5000)] = k
    while b.pending:
        for slot, z, gap, it, conv in b.run(steps=8):
            res[owner.pop(slot)] = (z, gap, it, conv)
    for k in range(len(imgs)):
        z, gap, it, conv = res[k]
        assert torch.equal(z, alone[k][0]) and it == alone[k][2] and gap == alone[k][1], SHAPES[k]


def test_bounded_runs_give_the_same_results(cuda):
    """max_chunks = 1: each run takes one chunk and may finish nothing; the
    images' results are the same bits as with unbounded runs."""
    import torch
    from fastprox_b200.batch import RaggedBatch
    imgs = _images(cuda)
    b = RaggedBatch(max_images=16, max_pixels=200_000)
    slots = [b.admit(x, g, t, max_iter=5000) for x, g, t in imgs]
    ref = _run_all(b)
    ref = [ref[s] for s in slots]
    b = RaggedBatch(max_images=16, max_pixels=200_000)
    owner = {b.admit(x, g, t, max_iter=5000): k for k, (x, g, t) in enumerate(imgs)}
    res, empty_runs = {}, 0
    while b.pending:
        out = b.run(steps=8, max_chunks=1)
        empty_runs += not out
        for slot, z, gap, it, conv in out:
            res[owner.pop(slot)] = (z, gap, it, conv)
    assert empty_runs > 0
    for k in range(len(imgs)):
        assert torch.equal(res[k][0], ref[k][0]) and res[k][1:] == ref[k][1:], SHAPES[k]
