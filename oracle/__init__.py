"""Test infrastructure: the checker for the image-TV path, never the product.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package. Nothing under ``fastprox_b200/`` does, and the
product path fails loudly rather than falling back to anything here.

Two independent checkers live here:

* ``ref_capi`` -- ctypes bindings to the reference fastprox C library, built
  from the reference's own sources by ``oracle/Makefile`` into
  ``oracle/_ref/libfastprox_ref.so`` (git-ignored; it travels with the tree).
  Its ``tv_iso`` / ``tv_aniso`` outputs, iteration counts and per-image gaps
  are the parity target.
* ``tv_np`` -- a NumPy FP64 restatement of the reference's isotropic dual
  FISTA (``src/ops/tv_iso.cpp:424-543``) and its anisotropic ADBPG / FDPG-3
  with the polish (``src/ops/tv_aniso.cpp:429-616, 886-953``), plus exact
  1D TV (Condat's direct algorithm).  Pinned against the CVXPY golden
  vectors in ``tests/golden/cvxpy_images.npz`` and against ``ref_capi``.
"""
