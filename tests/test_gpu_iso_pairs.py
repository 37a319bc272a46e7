"""Several isotropic iterations in one launch against the same iterations
one launch each.

Pairs (iso2d_pair_kernel: iterations 1 and 2 mod 4, and 3 and 4 mod 4 with
the gap check and restart test in the second) against single steps: the same
arithmetic per iteration and the same order of every sum, so the same
iterates, iteration counts and gaps, bit for bit. Quads (iso2d_quad_kernel:
iterations 1 to 4 mod 4, the fourth with the check) against pairs: the same
arithmetic per iteration, so the same iterates and duals bit for bit and the
same iteration counts; their gap and restart sums are formed in an order of
their own (per row and warp strip), so the gaps agree to rounding.
Covers images with and without pixel weights, heights that leave blocks of 4
to 12 rows and a last block shorter than the rest, images of two and three
rows, widths below the block's 512 columns, widths above it (several column
blocks or strips; the halo columns), per-image steps (images that stop at
different iterations), warm starts, and max_iter values that end inside a
pair or a quad. The float64 cases run single steps either way (pairs and
quads are float32 paths) and check that the switches leave them alone. Each
arm is a child process with its switch in the environment
(FASTPROX_B200_PAIRS=0: single steps only; FASTPROX_B200_QUADS=0: no quads;
the library reads its tuning hints once)."""

import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]

CASES = [  # (dtype, B, H, W, alpha, tol, max_iter, warm)
    (np.float32, 3, 512, 512, True, 1e-6, 400, False),
    (np.float32, 2, 37, 100, False, 1e-7, 500, False),
    (np.float64, 3, 130, 256, True, 1e-9, 2000, False),
    (np.float64, 2, 5, 64, False, 0.0, 6, False),
    (np.float32, 2, 64, 508, True, 0.0, 7, False),
    (np.float64, 2, 96, 128, False, 1e-8, 3000, True),
    (np.float32, 3, 2, 40, True, 1e-7, 300, False),
    (np.float32, 2, 3, 36, False, 0.0, 9, False),
    (np.float32, 2, 40, 1024, True, 1e-7, 400, False),
    (np.float32, 2, 33, 640, False, 0.0, 9, False),
    (np.float32, 2, 29, 1540, True, 1e-6, 300, True),
]


def _run(i):
    import torch
    from fastprox_b200 import TVIso, synth
    dtype, B, H, W, alpha, tol, max_iter, warm = CASES[i]
    x = synth.phantom(B, H, W, seed=70 + i).astype(dtype)
    al = synth.pixel_weights((H, W), seed=80 + i).astype(np.float64) if alpha else None
    op = TVIso(2, pixel_weights=al)
    steps = torch.as_tensor(np.linspace(0.05, 0.2, B), device="cuda")
    xt = torch.as_tensor(x, device="cuda")
    dual = None
    if warm:  # a warm start from a loose solve of the same images
        _, info0 = op.solve(xt, steps, tol=1e-3, max_iter=200)
        dual = info0.dual
    z, info = op.solve(xt, steps, tol=tol, max_iter=max_iter, warm=warm, dual=dual)
    torch.cuda.synchronize()
    # the dual too: where a checked pair passed, its first iterate is formed again
    q = info.dual.cpu().numpy() if hasattr(info.dual, "cpu") else np.asarray(info.dual)
    return z.cpu().numpy(), np.asarray(info.image_iters), np.asarray(info.gaps), q


def _arm(tmp_path, name, **env):
    out = tmp_path / f"{name}.npz"
    r = subprocess.run([sys.executable, str(pathlib.Path(__file__)), str(out)], cwd=ROOT,
                       env=dict(os.environ, **env), capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    return np.load(out)


@pytest.mark.gpu
def test_pairs_match_single_steps(cuda, tmp_path):
    ref = _arm(tmp_path, "single", FASTPROX_B200_PAIRS="0")
    got = _arm(tmp_path, "pairs", FASTPROX_B200_QUADS="0")
    for i in range(len(CASES)):
        assert np.array_equal(got[f"it{i}"], ref[f"it{i}"]), (i, got[f"it{i}"], ref[f"it{i}"])
        assert np.array_equal(got[f"z{i}"], ref[f"z{i}"]), (i, np.abs(got[f"z{i}"] - ref[f"z{i}"]).max())
        assert np.array_equal(got[f"g{i}"], ref[f"g{i}"]), (i, got[f"g{i}"], ref[f"g{i}"])
        assert np.array_equal(got[f"q{i}"], ref[f"q{i}"]), (i, np.abs(got[f"q{i}"] - ref[f"q{i}"]).max())


@pytest.mark.gpu
def test_quads_match_pairs(cuda, tmp_path):
    ref = _arm(tmp_path, "pairs", FASTPROX_B200_QUADS="0")
    for i in range(len(CASES)):
        z, iters, gaps, q = _run(i)
        assert np.array_equal(iters, ref[f"it{i}"]), (i, iters, ref[f"it{i}"])
        assert np.array_equal(z, ref[f"z{i}"]), (i, np.abs(z - ref[f"z{i}"]).max())
        assert np.array_equal(q, ref[f"q{i}"]), (i, np.abs(q - ref[f"q{i}"]).max())
        np.testing.assert_allclose(gaps, ref[f"g{i}"], rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_step_timing_counts_launch_kinds(cuda):
    """fp_b200_workspace_time_steps: 12 iterations of a batch that never
    converges run as a cold single step, quads at iterations 1 and 5, a pair
    at 9 (a quad would cross max_iter), and single steps at 11 and 12 (the
    check at max_iter); with quads off, pairs at 1, 5, 9, pairs with the check
    at 3 and 7, and single steps from 11 on (a child process)."""
    import ctypes as C

    import torch
    from fastprox_b200 import TVIso, capi, synth
    L = capi.lib()
    x = torch.as_tensor(synth.phantom(4, 64, 128, seed=90), device=cuda)
    op = TVIso(2)
    ws = op.workspace(x)
    capi.check(L.fp_b200_workspace_time_steps(ws, 1), "time_steps")
    op.solve(x, 0.1, tol=0.0, max_iter=12, with_dual=False)
    ms, n = C.c_double(), C.c_int64()
    got = []
    for kind in range(4):
        capi.check(L.fp_b200_workspace_step_times(ws, kind, C.byref(ms), C.byref(n)), "step_times")
        got.append((n.value, ms.value))
    # (launches past the last iteration, in the chunk the host issues before it
    # reads that every image stopped, are single steps that exit at once)
    assert got[3][0] == 2 and got[1][0] == 1 and got[2][0] == 0 and got[0][0] >= 3, got
    assert got[3][1] > 0.0 and got[0][1] > 0.0, got
    capi.check(L.fp_b200_workspace_time_steps(ws, 0), "time_steps")
    op.solve(x, 0.1, tol=0.0, max_iter=12, with_dual=False)
    capi.check(L.fp_b200_workspace_step_times(ws, 3, C.byref(ms), C.byref(n)), "step_times")
    assert n.value == 0
    assert L.fp_b200_workspace_step_times(ws, 4, None, None) == capi.FP_EINVAL
    r = subprocess.run([sys.executable, "-c", _KINDS_NO_QUADS, str(ROOT)], cwd=ROOT,
                       env=dict(os.environ, FASTPROX_B200_QUADS="0"), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


_KINDS_NO_QUADS = r"""
import ctypes as C, sys
sys.path.insert(0, sys.argv[1])
import torch
from fastprox_b200 import TVIso, capi, synth
L = capi.lib()
x = torch.as_tensor(synth.phantom(4, 64, 128, seed=90), device="cuda")
op = TVIso(2)
ws = op.workspace(x)
capi.check(L.fp_b200_workspace_time_steps(ws, 1), "time_steps")
op.solve(x, 0.1, tol=0.0, max_iter=12, with_dual=False)
ms, n = C.c_double(), C.c_int64()
got = []
for kind in range(4):
    capi.check(L.fp_b200_workspace_step_times(ws, kind, C.byref(ms), C.byref(n)), "step_times")
    got.append(n.value)
assert got[1] == 3 and got[2] == 2 and got[0] >= 3 and got[3] == 0, got
"""


if __name__ == "__main__":  # one arm (its switches in the environment)
    sys.path.insert(0, str(ROOT))
    res = {}
    for i in range(len(CASES)):
        z, it, g, q = _run(i)
        res.update({f"z{i}": z, f"it{i}": it, f"g{i}": g, f"q{i}": q})
    np.savez(sys.argv[1], **res)
