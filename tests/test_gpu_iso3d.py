"""The 3D isotropic step in its two forms: two voxels per thread (the default
for float32 volumes whose rows have an even number of voxels: 64 x 8 tiles,
8-byte staging copies) and one voxel per thread (FASTPROX_B200_3D_V2=0,
32 x 8 tiles). Both run the same per-voxel arithmetic; their gap and restart
sums run in orders of their own, so their iterates agree to rounding and
their iteration counts to a check or two. The volumes span several tiles in
every axis, a partial tile among them, and carry pixel weights; the two-voxel
form is also checked against the reference library. The one-voxel form runs
in a child process (the library reads its tuning hints once)."""

import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
SHAPES = [(12, 18, 150), (9, 33, 64), (5, 8, 10)]


def _run(shape, tol, max_iter):
    import torch
    from fastprox_b200 import TVIso, synth
    x = synth.phantom3d(2, *shape, seed=31)
    al = synth.pixel_weights(shape, seed=32)
    z, info = TVIso(3, pixel_weights=al).solve(torch.as_tensor(x, device="cuda"), np.array([0.06, 0.15]), tol=tol,
                                              max_iter=max_iter)
    torch.cuda.synchronize()
    return x, al, z.cpu().numpy(), np.asarray(info.image_iters)


def _nrel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
def test_two_voxel_step_against_reference(cuda, shape):
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built")
    x, al, z, iters = _run(shape, 1e-6, 100000)
    for i, g in enumerate((0.06, 0.15)):
        r = ref_capi.solve(x[i:i + 1], g, iso=True, k=3, spatial=al, tol=1e-6, max_iter=100000)
        assert _nrel(z[i], r.z[0]) <= 1e-5, (shape, i, _nrel(z[i], r.z[0]))
        itr = int(r.iters[0])
        assert abs(int(iters[i]) - itr) <= max(4, 0.2 * itr), (shape, i, iters[i], itr)


@pytest.mark.gpu
def test_two_voxel_step_against_one_voxel_step(cuda, tmp_path):
    out = tmp_path / "one.npz"
    r = subprocess.run([sys.executable, str(pathlib.Path(__file__)), str(out)], cwd=ROOT,
                       env=dict(os.environ, FASTPROX_B200_3D_V2="0"), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    one = np.load(out)
    for k, shape in enumerate(SHAPES):
        # a fixed iteration count (tol 0): the same iterations on both sides
        _, _, z, _ = _run(shape, 0.0, 40)
        assert np.abs(z - one[f"z{k}"]).max() <= 1e-6 * (1.0 + np.abs(z).max()), shape
        # to the gap: the same certified accuracy, counts within a check or two
        _, _, z, iters = _run(shape, 1e-6, 100000)
        assert _nrel(z, one[f"zt{k}"]) <= 1e-5, shape
        assert np.all(np.abs(iters - one[f"it{k}"]) <= 8), (shape, iters, one[f"it{k}"])


if __name__ == "__main__":  # the one-voxel form (its switch in the environment)
    sys.path.insert(0, str(ROOT))
    res = {}
    for k, shape in enumerate(SHAPES):
        res[f"z{k}"] = _run(shape, 0.0, 40)[2]
        _, _, res[f"zt{k}"], res[f"it{k}"] = _run(shape, 1e-6, 100000)
    np.savez(sys.argv[1], **res)
