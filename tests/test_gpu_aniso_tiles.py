"""The tiled fibre passes of anisotropic TV (a block's fibres in shared
memory, scanned by one warp in lockstep) against the untiled passes (one
thread per fibre over global memory), which run the same arithmetic: a few
iterations of each on the same inputs give the same iterates. Fibres of every
kind share a warp: ordinary ones, constant ones (their own prox), ones with a
zero-weight edge (independent pieces) and, without edge weights, steps large
enough that a fibre's prox is its mean. The untiled run is a child process
with FASTPROX_B200_TILES=0 (the library reads its tuning hints once)."""

import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _inputs(dtype, edge):
    from fastprox_b200 import synth
    x = synth.phantom(3, 72, 130, seed=61).astype(dtype)
    x[0, 5, :] = 0.3    # a constant row
    x[1, :, 7] = 0.5    # a constant column
    beta = None
    if edge:
        beta = synth.pixel_weights((2, 72, 130), seed=62).astype(dtype)
        beta[0, 10, 20] = 0.0   # zero-weight edges: their fibres fall in pieces
        beta[1, 30, 40] = 0.0
        beta[0, 50, :] = 0.0    # a row of them
    steps = np.array([0.05, 0.1, 50.0])
    return x, beta, steps


def _run(dtype, edge, iters):
    import torch
    from fastprox_b200 import TVAniso
    x, beta, steps = _inputs(dtype, edge)
    op = TVAniso(2, edge_weights=beta)
    z, info = op.solve(torch.as_tensor(x, device="cuda"), torch.as_tensor(steps, device="cuda"), tol=0.0,
                       max_iter=iters, with_dual=False)
    torch.cuda.synchronize()
    return z.cpu().numpy()


CASES = [(np.float64, False), (np.float64, True), (np.float32, False), (np.float32, True)]


@pytest.mark.gpu
@pytest.mark.parametrize("iters", [1, 6])
def test_tiled_passes_match_untiled(cuda, tmp_path, iters):
    env = dict(os.environ, FASTPROX_B200_TILES="0")
    out = tmp_path / "untiled.npz"
    r = subprocess.run([sys.executable, str(pathlib.Path(__file__)), str(out), str(iters)], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = np.load(out)
    for i, (dtype, edge) in enumerate(CASES):
        z = _run(dtype, edge, iters)
        zu = ref[f"z{i}"]
        assert z.dtype == zu.dtype
        scale = 1.0 + np.abs(zu).max()
        # the same arithmetic: equal up to the order of the restart test's sums
        tol = 1e-13 if dtype == np.float64 else 1e-6
        assert np.abs(z - zu).max() <= tol * scale, (dtype, edge, np.abs(z - zu).max())


if __name__ == "__main__":  # the untiled run (FASTPROX_B200_TILES=0 in the environment)
    sys.path.insert(0, str(ROOT))
    n = int(sys.argv[2])
    np.savez(sys.argv[1], **{f"z{i}": _run(dt, e, n) for i, (dt, e) in enumerate(CASES)})
