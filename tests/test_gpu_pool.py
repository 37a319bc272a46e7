"""Workspaces from the library's memory pool: many created and freed in a
row, of changing shapes and kinds, on several streams at once, give the
results of a fresh solve; fp_b200_release_cached returns the memory and
later solves still work."""

import concurrent.futures as cf

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _nrel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _cases(cuda):
    import torch
    from fastprox_b200 import synth
    out = []
    for i, (h, w) in enumerate([(64, 64), (96, 40), (128, 200), (33, 37), (256, 256), (64, 64)]):
        x = torch.as_tensor(synth.phantom(1, h, w, seed=10 + i)[0], device=cuda)
        out.append((i % 2 == 0, x, 0.05 + 0.02 * i))
    return out


def _solve(iso, x, g):
    from fastprox_b200 import TVAniso, TVIso
    op = TVIso(2) if iso else TVAniso(2)
    z, info = op.solve(x[None], g, tol=1e-5, max_iter=3000, with_dual=False)
    return z[0], info.image_iters[0]


def test_reused_workspaces_and_streams(cuda):
    import torch
    from fastprox_b200 import capi
    cases = _cases(cuda)
    ref = [_solve(*c) for c in cases]
    torch.cuda.synchronize()
    for _ in range(3):
        for c, (zr, itr) in zip(cases, ref):
            z, it = _solve(*c)
            assert torch.equal(z, zr) and it == itr
    streams = [torch.cuda.Stream() for _ in range(3)]

    def work(k):
        s = streams[k % 3]
        s.wait_stream(torch.cuda.default_stream())
        with torch.cuda.stream(s):
            z, it = _solve(*cases[k % len(cases)])
            s.synchronize()
        return k, z, it

    with cf.ThreadPoolExecutor(3) as ex:
        for k, z, it in ex.map(work, range(12)):
            zr, itr = ref[k % len(cases)]
            assert torch.equal(z, zr) and it == itr, k
    capi.lib().fp_b200_release_cached()
    z, it = _solve(*cases[2])
    assert _nrel(z, ref[2][0]) == 0.0 and it == ref[2][1]


def test_prox_with_a_workspace_reserves_no_device_memory(cuda):
    """The reference's rule that a prox call given a workspace allocates
    nothing (its allocation counter, tests/c/test_core.cpp:40-66; device rule
    docs/spec.md:887): after the workspace exists and one call has run (the
    library's kernels loaded), further calls, isotropic and anisotropic, with
    one step or one per image, leave the device's free memory unchanged."""
    import torch
    from fastprox_b200 import TVAniso, TVIso, synth
    x = torch.as_tensor(synth.phantom(3, 96, 128, seed=50), device=cuda)
    steps = torch.tensor([0.05, 0.1, 0.2], dtype=torch.float64, device=cuda)
    ops = [TVIso(2), TVAniso(2), TVIso(2, pixel_weights=synth.pixel_weights((96, 128), seed=51))]
    out = torch.empty_like(x)
    for op in ops:
        op.solve(x, 0.1, tol=1e-5, max_iter=2000, out=out, with_dual=False)
        op.solve(x, steps, tol=1e-5, max_iter=2000, out=out, with_dual=False)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        for op in ops:
            op.solve(x, 0.1, tol=1e-5, max_iter=2000, out=out, with_dual=False)
            op.solve(x, steps, tol=1e-5, max_iter=2000, out=out, with_dual=False)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
