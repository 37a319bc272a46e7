"""The fibre passes of anisotropic TV in their three forms, which run the
same arithmetic, against each other: the fibre-major passes (the default: a
lane per fibre over a fibre-major copy of the fibres, every fibre of the
launch in flight), the tiled passes (a block's fibres in shared memory,
scanned by one warp in lockstep; FASTPROX_B200_AN_FIB=0) and the untiled
passes (one thread per fibre over global memory; also
FASTPROX_B200_TILES=0). A few iterations of each on the same inputs give the
same iterates, up to the order of the restart test's sums. Fibres of every
kind share a warp: ordinary ones, constant ones (their own prox), ones with a
zero-weight edge (independent pieces) and, without edge weights, steps large
enough that a fibre's prox is its mean. The other forms run in child
processes (the library reads its tuning hints once)."""

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


def _arm(tmp_path, name, iters, **env):
    out = tmp_path / f"{name}.npz"
    r = subprocess.run([sys.executable, str(pathlib.Path(__file__)), str(out), str(iters)], cwd=ROOT,
                       env=dict(os.environ, **env), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.load(out)


def _close(z, zu, dtype, what):
    assert z.dtype == zu.dtype
    scale = 1.0 + np.abs(zu).max()
    # the same arithmetic: equal up to the order of the restart test's sums
    tol = 1e-13 if dtype == np.float64 else 1e-6
    assert np.abs(z - zu).max() <= tol * scale, (what, dtype, np.abs(z - zu).max())


@pytest.mark.gpu
@pytest.mark.parametrize("iters", [1, 6])
def test_fibre_pass_forms_agree(cuda, tmp_path, iters):
    untiled = _arm(tmp_path, "untiled", iters, FASTPROX_B200_AN_FIB="0", FASTPROX_B200_TILES="0")
    tiled = _arm(tmp_path, "tiled", iters, FASTPROX_B200_AN_FIB="0")
    for i, (dtype, edge) in enumerate(CASES):
        z = _run(dtype, edge, iters)
        _close(z, untiled[f"z{i}"], dtype, ("fibre-major", edge))
        _close(tiled[f"z{i}"], untiled[f"z{i}"], dtype, ("tiled", edge))


if __name__ == "__main__":  # one form (its switches in the environment)
    sys.path.insert(0, str(ROOT))
    n = int(sys.argv[2])
    np.savez(sys.argv[1], **{f"z{i}": _run(dt, e, n) for i, (dt, e) in enumerate(CASES)})
