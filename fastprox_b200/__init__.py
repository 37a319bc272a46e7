"""fastprox_b200: fastprox's image total-variation prox (isotropic and
anisotropic, 2D and 3D, by dual FISTA stopped on the duality gap) on NVIDIA
B200 (sm_100a), behind the reference's plain-C ABI (include/fastprox_b200.h).

* ``capi``      -- ctypes bindings to libfastprox_b200.so
* ``image_tv``  -- TVIso / TVAniso operator objects (NumPy and torch arrays), and
  TVIsoHuber / TVAnisoHuber (Huber-smoothed TV)
* ``torch``     -- the PyTorch wrapper (tv_iso / tv_aniso with autograd)
* ``synth``     -- seeded synthetic images (phantoms, noise)
* ``build``     -- builds the shared library in-tree
"""

from .capi import FastproxError, LIB_PATH  # noqa: F401
from .image_tv import IterInfo, TVAniso, TVAnisoHuber, TVIso, TVIsoHuber, tv_aniso, tv_iso  # noqa: F401

__all__ = ["TVIso", "TVAniso", "TVIsoHuber", "TVAnisoHuber", "tv_iso", "tv_aniso", "IterInfo", "FastproxError",
           "LIB_PATH"]
