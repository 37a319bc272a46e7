"""Ragged batches of isotropic 2D TV (fp_b200_batch_* in the C ABI): images of
mixed sizes solved in one set of launches, each to its own step and
tolerance, with images admitted while others iterate (continuous batching).

    b = RaggedBatch(max_images=256, max_pixels=80_000_000)
    slots = [b.admit(x_i, gamma_i, tol_i, out=z_i) for ...]   # CUDA tensors
    while b.pending: finished = b.run()                        # [(slot, gap, iters)]
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .image_tv import TVIso


class RaggedBatch:
    def __init__(self, max_images, max_pixels, dtype="float32", weights=None, rows=0, stream=None, graphs=True,
                 quads=True, quad_rows=0):
        import torch
        self.op = TVIso(2, weights)
        self.max_images = int(max_images)
        self._h = C.c_void_p()
        dt = capi.FP_F32 if str(dtype).endswith("float32") else capi.FP_F64
        capi.check(capi.lib().fp_b200_batch_create(self.op._op, self.max_images, int(max_pixels), dt,
                                                    C.byref(self._h)), "batch_create")
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        capi.check(capi.lib().fp_b200_batch_set_stream(self._h, C.c_void_p(s)), "batch_stream")
        if rows:
            capi.check(capi.lib().fp_b200_batch_set_rows(self._h, int(rows)), "batch_rows")
        if not graphs:
            capi.check(capi.lib().fp_b200_batch_set_graphs(self._h, 0), "batch_graphs")
        capi.check(capi.lib().fp_b200_batch_set_quads(self._h, int(bool(quads)), int(quad_rows)), "batch_quads")
        self.pending = 0
        self._keep = {}
        self._fin = np.zeros(self.max_images, np.int32)
        self._gaps = np.zeros(self.max_images)
        self._its = np.zeros(self.max_images, np.int32)

    def __del__(self):
        try:
            if self._h:
                capi.lib().fp_b200_batch_free(self._h)
        except Exception:
            pass

    def admit(self, x, gamma, tol=1e-6, max_iter=1000, out=None):
        """Admits one (H, W) CUDA tensor; returns its slot, or None when the
        batch is full (run, then admit again)."""
        import torch
        x = x.contiguous()
        z = torch.empty_like(x) if out is None else out
        slot = C.c_int(-1)
        st = capi.lib().fp_b200_batch_admit(self._h, C.c_void_p(x.data_ptr()), x.shape[-2], x.shape[-1],
                                            float(gamma), float(tol), int(max_iter), C.c_void_p(z.data_ptr()),
                                            C.byref(slot))
        if st == capi.FP_ENOMEM:
            return None
        capi.check(st, "batch_admit")
        self._keep[slot.value] = (x, z)
        self.pending += 1
        return slot.value

    def run(self, steps=8, max_chunks=0):
        """Iterates until some images finish (or, with max_chunks > 0, at most
        that many chunks of `steps` steps; a step advances each live image by
        one iteration, or by four where the pair variants take it); returns
        [(slot, z, gap, iters, converged)]."""
        nf, nl = C.c_int(0), C.c_int(0)
        capi.check(capi.lib().fp_b200_batch_run(self._h, int(steps), int(max_chunks),
                                                self._fin.ctypes.data_as(C.POINTER(C.c_int)),
                                                self._gaps.ctypes.data_as(C.POINTER(C.c_double)),
                                                self._its.ctypes.data_as(C.POINTER(C.c_int)), C.byref(nf),
                                                C.byref(nl)), "batch_run")
        out = []
        for i in range(nf.value):
            slot = int(self._fin[i])
            x, z = self._keep.pop(slot)
            it = int(self._its[i])
            out.append((slot, z, float(self._gaps[i]), abs(it), it >= 0))
        self.pending -= nf.value
        return out

    def stats(self):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        capi.lib().fp_b200_batch_stats(self._h, C.byref(a), C.byref(b), C.byref(c))
        return {"kernel_launches": a.value, "steps": b.value, "free_pixels": c.value}
