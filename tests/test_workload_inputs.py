"""The workloads' seeded synthetic inputs against the configurations they
stand for (no GPU): the benchmark batch (64 phantoms of 512 x 512 with noise
0.1, a pixel-weight map U[0.5, 1.5], steps cycling 0.05 / 0.1 / 0.2), the
uneven batch (256 images, sides from {64, 96, ..., 1024}, steps
log-uniform in [0.01, 0.5], tolerances log-uniform in [1e-6, 1e-4]) and the
serving stream (Poisson arrivals at 200 per second, half isotropic and half
anisotropic 2D with sides log-uniform in [64, 2048], 5 % 128^3 volumes,
steps log-uniform in [0.02, 0.3], tolerance 1e-5). Seeded: the same inputs
on every run and every machine."""

import math
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def test_benchmark_batch():
    import bench
    x, alpha, steps = bench.make_inputs()
    assert x.shape == (64, 512, 512) and x.dtype == np.float32
    assert alpha.shape == (512, 512) and alpha.min() >= 0.5 and alpha.max() <= 1.5
    assert list(steps[:6]) == [0.05, 0.1, 0.2, 0.05, 0.1, 0.2]
    # piecewise-constant intensities in [0, 1] plus N(0, 0.1^2): the noise's spread
    # shows around the phantom's levels
    assert -1.0 < float(x.min()) < 0.0 and 1.0 < float(x.max()) < 2.0
    x2, _, _ = bench.make_inputs()
    assert np.array_equal(x, x2)


def test_uneven_batch_specification(monkeypatch):
    from fastprox_b200 import synth, workloads
    # the images themselves are phantoms of the listed shapes; skip drawing them
    monkeypatch.setattr(synth, "phantom", lambda b, h, w, seed=0, **k: np.zeros((b, h, w), np.float32))
    shapes, gammas, tols, imgs = workloads._uneven_inputs()
    assert len(shapes) == len(gammas) == len(tols) == len(imgs) == 256
    sides = {s for hw in shapes for s in hw}
    assert sides <= set(range(64, 1025, 32)) and min(sides) == 64 and max(sides) == 1024
    assert any(h != w for h, w in shapes)  # height and width drawn independently
    assert 0.01 <= gammas.min() and gammas.max() <= 0.5
    assert 1e-6 <= tols.min() and tols.max() <= 1e-4
    # log-uniform: about half below the geometric midpoint
    assert 0.35 < np.mean(gammas < math.sqrt(0.01 * 0.5)) < 0.65
    assert 0.35 < np.mean(tols < 1e-5) < 0.65


def test_serving_stream_specification():
    from fastprox_b200 import serve
    reqs = serve.make_requests(60.0, 200.0, 0)
    n = len(reqs)
    assert abs(n - 12000) < 4 * math.sqrt(12000)  # Poisson(200/s) over 60 s
    ts = np.array([r.t for r in reqs])
    assert np.all(np.diff(ts) > 0) and ts[-1] < 60.0
    kinds = [r.kind for r in reqs]
    f3 = kinds.count("iso3d") / n
    assert 0.04 < f3 < 0.06
    iso, an = kinds.count("iso2d"), kinds.count("aniso2d")
    assert abs(iso - an) < 4 * math.sqrt(iso + an)
    for r in reqs:
        assert 0.02 <= r.gamma <= 0.3 and r.tol == 1e-5
        if r.kind == "iso3d":
            assert r.side == 128
        else:
            assert 64 <= r.side <= 2048
    sides = np.array([r.side for r in reqs if r.kind != "iso3d"], float)
    assert 0.4 < np.mean(sides < math.sqrt(64 * 2048)) < 0.6  # log-uniform
    # seeded: the same stream again
    again = serve.make_requests(60.0, 200.0, 0)
    assert [(r.t, r.kind, r.side, r.gamma) for r in again] == [(r.t, r.kind, r.side, r.gamma) for r in reqs]
