"""Loaders of the committed golden fixtures (tests/golden/)."""

import pathlib

import numpy as np

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def _group(path):
    data = np.load(path)
    out = {}
    for key in data.files:
        name, fieldname = key.split("/", 1)
        out.setdefault(name, {"param": {}})
        if fieldname.startswith("param/"):
            out[name]["param"][fieldname[6:]] = data[key]
        else:
            out[name][fieldname] = data[key]
    return out


def cvxpy_problems():
    """The reference's CVXPY/Clarabel image-TV problems, in key order."""
    probs = _group(GOLDEN / "cvxpy_images.npz")
    return [probs[k] for k in sorted(probs)]


def ref_vectors():
    """name -> dict of the reference C library's outputs on seeded inputs."""
    return _group(GOLDEN / "ref_vectors.npz")
