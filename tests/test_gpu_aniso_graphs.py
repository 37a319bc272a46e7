"""Small anisotropic solves replay their rounds as captured CUDA graphs
(chunks of rounds, captured again when the live list shrinks or the call's
constants change); the same solves in plain launches give the same bits:
iterates, iteration counts and gaps. Covers 2D (ADBPG) and 3D (FDPG-3),
float32 and float64, edge weights, per-image steps (images that stop at
different rounds, so the live list shrinks), a warm start, and two calls on
one operator with different tolerances (the second replays or recaptures).
The plain run is a child process with FASTPROX_B200_AN_GRAPHS=0 (the library
reads its tuning hints once)."""

import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _cases():
    from fastprox_b200 import synth
    out = []
    x = synth.phantom(3, 40, 52, seed=5)
    beta = synth.pixel_weights((2, 40, 52), seed=6)
    out.append(("2d", x.astype(np.float32), None, [0.05, 0.1, 0.3], 1e-6, 2000, False))
    out.append(("2d", x.astype(np.float64), beta, [0.05, 0.2, 0.1], 1e-8, 3000, False))
    out.append(("2d", x[:1].astype(np.float32), None, [0.1], 1e-6, 2000, True))
    v = synth.phantom3d(2, 12, 14, 16, seed=7)
    out.append(("3d", v.astype(np.float32), None, [0.05, 0.2], 1e-5, 2000, False))
    out.append(("3d", v.astype(np.float64), None, [0.1, 0.1], 1e-8, 3000, False))
    return out


def _run():
    import torch
    from fastprox_b200 import TVAniso
    res = []
    for kind, x, beta, steps, tol, max_iter, warm in _cases():
        op = TVAniso(2 if kind == "2d" else 3, edge_weights=beta)
        xt = torch.as_tensor(x, device="cuda")
        st = torch.as_tensor(np.asarray(steps, dtype=np.float64), device="cuda")
        dual = None
        if warm:  # a warm start from a loose solve
            _, info0 = op.solve(xt, st, tol=1e-3, max_iter=200)
            dual = info0.dual
        for t in (tol, 10 * tol):  # two calls on one workspace
            z, info = op.solve(xt, st, tol=t, max_iter=max_iter, warm=warm, dual=dual)
            torch.cuda.synchronize()
            res.append((z.cpu().numpy(), np.asarray(info.image_iters), np.asarray(info.gaps)))
    return res


@pytest.mark.gpu
def test_graph_rounds_match_plain_launches(cuda, tmp_path):
    env = dict(os.environ, FASTPROX_B200_AN_GRAPHS="0")
    out = tmp_path / "plain.npz"
    r = subprocess.run([sys.executable, str(pathlib.Path(__file__)), str(out)], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = np.load(out)
    for i, (z, its, gaps) in enumerate(_run()):
        assert np.array_equal(z, ref[f"z{i}"]), (i, np.abs(z - ref[f"z{i}"]).max())
        assert np.array_equal(its, ref[f"i{i}"]), (i, its, ref[f"i{i}"])
        assert np.array_equal(gaps, ref[f"g{i}"]), (i, gaps, ref[f"g{i}"])


if __name__ == "__main__":  # the plain run (FASTPROX_B200_AN_GRAPHS=0 in the environment)
    sys.path.insert(0, str(ROOT))
    arrays = {}
    for i, (z, its, gaps) in enumerate(_run()):
        arrays[f"z{i}"], arrays[f"i{i}"], arrays[f"g{i}"] = z, its, gaps
    np.savez(sys.argv[1], **arrays)
