"""The serving loop on the GPU: a short Poisson stream of mixed requests
(isotropic and anisotropic 2D of mixed sizes, 3D volumes) served with
continuous batching; every request finishes, and each result is the same
alone and in the mix: a request solved by itself (one call) against its
result from the stream (isotropic 2D from the ragged batch, anisotropic and
3D from batches of requests of the same shape), within 1e-5 relative (the
float32 parity tolerance). Anisotropic and 3D requests of one shape batched
together against each solved alone, too."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _nrel(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_groups_match_single_requests(cuda):
    from fastprox_b200.serve import ImageSource, Request, solve_group
    src = ImageSource(3)
    for kind, side in (("aniso2d", 200), ("iso3d", 128)):
        reqs = [Request(i, 0.0, kind, side, g) for i, g in enumerate((0.05, 0.1, 0.2))]
        for r in reqs:
            r.x = src.image(r)
        zs, info = solve_group(reqs)
        assert info.converged
        for r, z in zip(reqs, zs):
            z1, _ = solve_group([r])
            assert _nrel(z, z1[0]) <= 1e-5, (kind, r.i, _nrel(z, z1[0]))


def test_short_stream_results_match_alone(cuda):
    from fastprox_b200.serve import ImageSource, make_requests, serve_stream, solve_group
    src = ImageSource(5)
    reqs = make_requests(1.5, rate=60.0, seed=7)
    kinds = {r.kind for r in reqs}
    assert {"iso2d", "aniso2d"} <= kinds
    lat, span = serve_stream(reqs, src, workers=4, keep=True)
    assert np.all(np.isfinite(lat)) and np.all(lat > 0)
    seen = {}
    for r in reqs:
        if seen.get(r.kind, 0) >= 3:
            continue
        seen[r.kind] = seen.get(r.kind, 0) + 1
        z1, _ = solve_group([r])
        assert _nrel(r.z, z1[0]) <= 1e-5, (r.kind, r.side, _nrel(r.z, z1[0]))
