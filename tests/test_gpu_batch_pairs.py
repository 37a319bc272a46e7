"""The ragged batch's pair variants (two iterations per launch on images with
rows of a multiple of 4 float pixels) against the same batch in single steps:
the same iterates, gaps and iteration counts, bit for bit (quads off in both).
Its quad launches (four iterations per launch) against pairs: the same
iterates and iteration counts, the gaps to rounding (their sums are formed
per quad tile). The images cover
one and several 512-column tiles across (the pair pass's halo columns at the
tile edges), a ragged last tile, a single row and widths off the 4-wide list
(single steps either way), per-image steps and tolerances, and max_iter values
that end inside a pair. The single-step run is a child process with
FASTPROX_B200_PAIRS=0 (the library reads its tuning hints once)."""

import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]

IMAGES = [  # (H, W, gamma, tol, max_iter)
    (64, 96, 0.1, 1e-6, 5000),
    (130, 1100, 0.05, 1e-5, 5000),
    (37, 1540, 0.2, 1e-6, 5000),
    (1, 80, 0.1, 1e-6, 5000),
    (33, 37, 0.1, 1e-6, 5000),
    (200, 32, 0.3, 1e-7, 5000),
    (48, 640, 0.1, 0.0, 7),
    (20, 512, 0.1, 0.0, 10),
]


def _run(rows, steps, quads=False):
    import torch
    from fastprox_b200 import synth
    from fastprox_b200.batch import RaggedBatch
    b = RaggedBatch(max_images=16, max_pixels=600_000, rows=rows, quads=quads)
    owner = {}
    for k, (h, w, g, t, mi) in enumerate(IMAGES):
        x = torch.as_tensor(synth.phantom(1, h, w, seed=90 + k)[0], device="cuda")
        owner[b.admit(x, g, t, max_iter=mi)] = k
    res = {}
    while b.pending:
        for slot, z, gap, it, conv in b.run(steps=steps):
            res[owner.pop(slot)] = (z.cpu().numpy(), gap, it, conv)
    torch.cuda.synchronize()
    return [res[k] for k in range(len(IMAGES))], b.stats()


CONFIGS = [(0, 8), (8, 4), (32, 3)]


@pytest.mark.gpu
def test_ragged_pairs_match_single_steps(cuda, tmp_path):
    env = dict(os.environ, FASTPROX_B200_PAIRS="0")
    out = tmp_path / "single.npz"
    r = subprocess.run([sys.executable, str(pathlib.Path(__file__)), str(out)], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = np.load(out)
    for c, (rows, steps) in enumerate(CONFIGS):
        res, stats = _run(rows, steps)
        for k, (z, gap, it, conv) in enumerate(res):
            zr = ref[f"z{c}_{k}"]
            gr, itr, cr = ref[f"m{c}_{k}"]
            assert np.array_equal(z, zr), (rows, IMAGES[k], np.abs(z - zr).max())
            assert it == int(itr) and bool(conv) == bool(cr), (rows, IMAGES[k], it, itr)
            assert gap == gr or (np.isnan(gap) and np.isnan(gr)), (rows, IMAGES[k], gap, gr)
        # the pair variants ran: three launches per step on the 4-wide list
        # (single steps and two pair variants), one on the other list
        assert stats["kernel_launches"] > 2 * stats["steps"], stats


@pytest.mark.gpu
def test_ragged_quads_match_pairs(cuda):
    for rows, steps in CONFIGS:
        ref, _ = _run(rows, steps, quads=False)
        got, stats = _run(rows, steps, quads=True)
        for k, ((z, gap, it, conv), (zr, gr, itr, cr)) in enumerate(zip(got, ref)):
            assert it == itr and conv == cr, (rows, IMAGES[k], it, itr)
            assert np.array_equal(z, zr), (rows, IMAGES[k], np.abs(z - zr).max())
            assert gap == gr or abs(gap - gr) <= 1e-12 * abs(gr) or (np.isnan(gap) and np.isnan(gr)), \
                (rows, IMAGES[k], gap, gr)


if __name__ == "__main__":  # the single-step run (FASTPROX_B200_PAIRS=0 in the environment)
    sys.path.insert(0, str(ROOT))
    arrays = {}
    for c, (rows, steps) in enumerate(CONFIGS):
        res, _ = _run(rows, steps)
        for k, (z, gap, it, conv) in enumerate(res):
            arrays[f"z{c}_{k}"] = z
            arrays[f"m{c}_{k}"] = np.array([gap, it, float(conv)])
    np.savez(sys.argv[1], **arrays)
