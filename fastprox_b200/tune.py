"""The autotuner of the ragged-batch engine: tile height (rows per block) and
steps per captured graph chunk (a step is one iteration of an image, or four
where the pair variants take it), chosen by timing short solves of the actual
batch and cached per shape class (in-process, and in
~/.cache/fastprox_b200/tune.json when that directory is writable). Longer
tuning solves (48 iterations) with chunks of 1 and 2 steps were measured and
not kept: they chose 2 steps, 1034 images/s on the uneven batch against 1057
with the 4 steps these choose; 64-row tiles were chosen when offered and ran
935 images/s against 1084 at 32 (short solves favour tiles that long ones,
with most images retired, cannot fill the SMs with).

A tuning solve runs 16 iterations (tol 0) of every image with each
candidate (tile height, steps per chunk, temporal-blocking depth); the
choice changes how work is tiled and how often the host polls, never the
iterations of an image (the same tiling is then used for every image of that
class, so results stay reproducible).
"""

from __future__ import annotations

import json
import math
import os
import pathlib
import time

ROWS = (8, 16, 32)
STEPS = (4, 8, 16)
DEPTHS = (2, 4)  # iterations per launch in steady state: pairs, or quads
_CACHE: dict = {}
_PATH = pathlib.Path(os.environ.get("FASTPROX_B200_TUNE", str(pathlib.Path.home() / ".cache" / "fastprox_b200"
                                                                / "tune.json")))


def shape_class(shapes):
    """The class of a batch: log2 of its median image size and of its count."""
    import numpy as np
    px = sorted(int(h) * int(w) for h, w in shapes)
    med = px[len(px) // 2]
    return f"m{int(math.log2(max(med, 1)))}_n{int(math.log2(max(len(px), 1)))}"


def _load():
    if not _CACHE and _PATH.exists():
        try:
            _CACHE.update(json.loads(_PATH.read_text()))
        except (OSError, ValueError):
            pass


def _save():
    try:
        _PATH.parent.mkdir(parents=True, exist_ok=True)
        _PATH.write_text(json.dumps(_CACHE, indent=1))
    except OSError:
        pass


def tune(images, max_pixels, retune=False):
    """images: [(x (H, W) CUDA tensor, gamma, tol)]. Returns {'rows', 'steps',
    'depth'}: the tile height, the steps per chunk, and the temporal-blocking
    depth (2: pair launches, 4: quad launches where the rows allow)."""
    import torch

    from .batch import RaggedBatch
    _load()
    key = shape_class([tuple(x.shape[-2:]) for x, _, _ in images]) + "_d"
    if key in _CACHE and not retune:
        return _CACHE[key]
    best, best_t = None, math.inf
    for depth in DEPTHS:
        for rows in ROWS:
            for steps in STEPS:
                b = RaggedBatch(len(images), max_pixels, rows=rows, quads=depth == 4)
                for x, g, _ in images:
                    b.admit(x, g, 0.0, max_iter=16)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                while b.pending:
                    b.run(steps=steps)
                torch.cuda.synchronize()
                t = time.perf_counter() - t0
                if t < best_t:
                    best, best_t = {"rows": rows, "steps": steps, "depth": depth}, t
                del b
    _CACHE[key] = best
    _save()
    return best
