"""The workloads besides the headline benchmark, each returning one JSON-able
dict (bench.py --workload NAME):

* ``aniso512``  anisotropic TV, 64 x 512^2 fp32 phantoms, gamma {0.05, 0.1, 0.2},
  gap <= 1e-6 (ADBPG with exact 1D steps and the polish on the device).
* ``uneven``    256 images, H and W uniform over {64, 96, ..., 1024}, phantom +
  noise, gamma log-uniform [0.01, 0.5], tol log-uniform [1e-6, 1e-4]: the
  ragged batch (tuned tiling, captured graphs) against the plain per-image
  loop of fp_prox calls.
* ``vjp``       (16, 3, 256, 256) fp32 phantom + noise(0.1), gamma 0.1, loss = MSE
  to the clean phantom: forward + implicit VJP time and memory against 400
  unrolled FISTA iterations in torch autograd; then (vjp_checks, on the
  first sample's three channels) the VJP against float64 central differences
  on 8 directions and the float32 gradient's error against the float64 one
  (tests/test_gpu_vjp.py checks it against the reference's fp_vjp).
* ``serve``     Poisson arrivals of denoising requests (see serve.py).
Seeded synthetic data throughout.
"""

from __future__ import annotations

import math
import time

import numpy as np


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def aniso512(args):
    import torch

    from . import synth
    from .image_tv import TVAniso
    B, H, W = 64, 512, 512
    x = torch.as_tensor(synth.phantom(B, H, W, seed=0), device="cuda")
    steps = torch.as_tensor([(0.05, 0.1, 0.2)[i % 3] for i in range(B)], device="cuda", dtype=torch.float64)
    # per-edge weights U[0.5, 1.5], one (2, H, W) map for the batch
    op = TVAniso(2, edge_weights=synth.pixel_weights((2, H, W), seed=1))
    out = torch.empty_like(x)
    for _ in range(max(args.warmup, 1)):
        z, info = op.solve(x, steps, tol=1e-6, max_iter=2000, out=out, with_dual=False)
    e0, e1 = _events()
    e0.record()
    for _ in range(args.steps):
        z, info = op.solve(x, steps, tol=1e-6, max_iter=2000, out=out, with_dual=False)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    return {"workload": "aniso512", "metric": "TV-prox images/s at gap<=1e-6 (512^2 fp32, anisotropic, edge weights)",
            "value": B / t, "unit": "images/s", "ms_per_step": t * 1e3, "converged": bool(info.converged),
            "iters": {"min": int(info.image_iters.min()), "median": float(np.median(info.image_iters)),
                      "max": int(info.image_iters.max())}}


def iso3d(args):
    """8 volumes of 128^3 float32 (phantom + noise 0.1), isotropic TV, gamma
    {0.05, 0.1, 0.2}, gap <= 1e-5 (the serving stream's volumes)."""
    import torch

    from . import synth
    from .image_tv import TVIso
    B, Dz, H, W = 8, 128, 128, 128
    x = torch.as_tensor(synth.phantom3d(B, Dz, H, W, seed=0), device="cuda")
    steps = torch.as_tensor([(0.05, 0.1, 0.2)[i % 3] for i in range(B)], device="cuda", dtype=torch.float64)
    op = TVIso(3)
    out = torch.empty_like(x)
    for _ in range(max(args.warmup, 1)):
        z, info = op.solve(x, steps, tol=1e-5, max_iter=20000, out=out, with_dual=False)
    e0, e1 = _events()
    e0.record()
    for _ in range(args.steps):
        z, info = op.solve(x, steps, tol=1e-5, max_iter=20000, out=out, with_dual=False)
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    vox_it = float(np.sum(info.image_iters)) * Dz * H * W
    return {"workload": "iso3d", "metric": "TV-prox volumes/s at gap<=1e-5 (128^3 fp32, isotropic)",
            "value": B / t, "unit": "volumes/s", "ms_per_step": t * 1e3, "converged": bool(info.converged),
            "iters": {"min": int(info.image_iters.min()), "median": float(np.median(info.image_iters)),
                      "max": int(info.image_iters.max())},
            "achieved_gbs": 52.0 * vox_it / t / 1e9, "bytes_per_voxel_iter": 52}


def _uneven_inputs(n=256, seed=0):
    from . import synth
    rng = np.random.default_rng(seed)
    sizes = np.arange(64, 1025, 32)
    shapes = [(int(rng.choice(sizes)), int(rng.choice(sizes))) for _ in range(n)]
    gammas = np.exp(rng.uniform(np.log(0.01), np.log(0.5), n))
    tols = np.exp(rng.uniform(np.log(1e-6), np.log(1e-4), n))
    imgs = [synth.phantom(1, h, w, seed=seed * 10007 + i)[0] for i, (h, w) in enumerate(shapes)]
    return shapes, gammas, tols, imgs


def uneven(args):
    import torch

    from . import tune
    from .batch import RaggedBatch
    from .image_tv import TVIso
    shapes, gammas, tols, imgs = _uneven_inputs()
    xs = [torch.as_tensor(im, device="cuda") for im in imgs]
    max_iter = 5000
    total_px = sum(h * w for h, w in shapes)
    cap = total_px + 4 * len(shapes)
    t0 = time.perf_counter()
    choice = tune.tune(list(zip(xs, gammas, tols)), cap)
    tune_s = time.perf_counter() - t0

    def ragged():
        b = RaggedBatch(len(xs), cap, rows=choice["rows"], quads=choice.get("depth", 4) == 4)
        outs = [torch.empty_like(x) for x in xs]
        e0, e1 = _events()
        e0.record()
        slots = [b.admit(x, g, t, max_iter=max_iter, out=o) for x, g, t, o in zip(xs, gammas, tols, outs)]
        res = {}
        while b.pending:
            for slot, z, gap, it, conv in b.run(steps=choice["steps"]):
                res[slot] = (it, conv)
        e1.record()
        torch.cuda.synchronize()
        st = b.stats()
        return e0.elapsed_time(e1) / 1e3, outs, [res[s] for s in slots], st

    ragged()  # warm-up (graphs captured)
    t_rag, outs, res, st = ragged()
    # the plain per-image loop: one fp_prox per image, workspaces created beforehand
    ops = [TVIso(2) for _ in xs]
    pouts = [torch.empty_like(x[None]) for x in xs]
    for op, x, po in zip(ops, xs, pouts):
        op.workspace(x[None])
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    infos = [op.solve(x[None], g, tol=t, max_iter=max_iter, out=po, with_dual=False)[1]
             for op, x, g, t, po in zip(ops, xs, gammas, tols, pouts)]
    e1.record()
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1) / 1e3
    errs = [float((o.double() - p[0].double()).norm() / p[0].double().norm()) for o, p in zip(outs, pouts)]
    pix_iters = sum(h * w * it for (h, w), (it, _) in zip(shapes, res))
    return {"workload": "uneven", "metric": "images/s, 256 mixed-size images (64..1024)^2, per-image gamma and tol",
            "value": len(xs) / t_rag, "unit": "images/s", "plain_loop_images_per_s": len(xs) / t_plain,
            "speedup_vs_plain": t_plain / t_rag, "seconds": t_rag, "plain_seconds": t_plain,
            "tuned": choice, "tune_seconds": tune_s, "converged": int(sum(c for _, c in res)),
            "max_rel_diff_vs_plain": max(errs), "achieved_GBs": 36 * pix_iters / t_rag / 1e9,
            "kernel_launches": st["kernel_launches"], "graph_steps": st["steps"], "pixels": total_px,
            # a seeded sample of the ragged results, for a comparison with the
            # reference (bench.py; not part of the printed line)
            "_sample": [(int(i), imgs[i], float(gammas[i]), float(tols[i]), outs[i].cpu().numpy(), int(res[i][0]))
                        for i in np.random.default_rng(5).choice(len(xs), 8, replace=False)]}


def vjp_checks(noisy, clean, gamma=0.1, ndir=32, h=1e-5, seed=1, tol64=1e-12):
    """The implicit VJP of the (B, C, H, W) workload's loss (MSE to the clean
    phantom) checked three ways, all in float64 on the GPU unless stated:
    * central differences: for ndir random unit directions d (seeded), the
      VJP's <gx, d> against (<g, z(x + h d)> - <g, z(x - h d)>) / 2h, g the
      loss's cotangent at z (and the same for gamma). Both sides run the same
      fixed number of iterations, twice those of the solve to gap tol64: a
      stop at different checks on the two sides would put the solver's own
      error, divided by 2h, into the difference. Each direction's error is
      relative to max(|<gx, d>|, 0.1 |gx| / sqrt(n)), a tenth of a random
      direction's typical derivative;
    * the float32 solve at gap 1e-6 and its VJP against the float64 one: the
      error of the float32 gradient, stated (its flat regions are read off an
      iterate certified to about 1e-3 relative, so small regions can differ).
    Returns the worst relative errors."""
    import torch

    from .image_tv import TVIso
    from .torch import tv_iso
    x64 = torch.as_tensor(noisy, device="cuda").double()
    c64 = torch.as_tensor(clean, device="cuda").double()
    n = x64.numel()

    def grads(x, c, tol, dtype):
        xr = x.to(dtype).clone().requires_grad_(True)
        g = torch.tensor(gamma, device="cuda", dtype=dtype, requires_grad=True)
        z = tv_iso(xr, g, tol=tol, max_iter=10 ** 6, deriv_tol=1e-12 if dtype == torch.float64 else None)
        loss = ((z - c.to(dtype)) ** 2).mean()
        loss.backward()
        return z.detach(), xr.grad.detach().double(), float(g.grad)

    z64, gx64, gg64 = grads(x64, c64, tol64, torch.float64)
    cot = 2.0 * (z64 - c64) / n  # d loss / dz at the float64 solution
    img = tuple(x64.shape[-2:])
    xb = x64.reshape((-1,) + img)
    cb = cot.reshape((-1,) + img)
    op = TVIso(2)
    fixed = 2 * op.solve(xb, gamma, tol=tol64, max_iter=10 ** 6, with_dual=False)[1].iters

    def fwd(xx, gam):
        return op.solve(xx, gam, tol=0.0, max_iter=fixed, with_dual=False)[0]

    rng = np.random.default_rng(seed)
    worst_fd = 0.0
    floor = 0.1 * float(gx64.norm()) / math.sqrt(n)
    for _ in range(ndir):
        d = torch.as_tensor(rng.normal(size=xb.shape), device="cuda")
        d = d / d.norm()
        fd = float(((fwd(xb + h * d, gamma) - fwd(xb - h * d, gamma)) * cb).sum()) / (2 * h)
        an = float((gx64.reshape(xb.shape) * d).sum())
        worst_fd = max(worst_fd, abs(fd - an) / max(abs(an), floor))
    fdg = float(((fwd(xb, gamma + h) - fwd(xb, gamma - h)) * cb).sum()) / (2 * h)
    err_gamma = abs(fdg - gg64) / max(abs(fdg), 1e-300)
    _, gx32, gg32 = grads(x64, c64, 1e-6, torch.float32)
    return {"fd_directions": ndir, "fd_h": h, "fd_max_rel_err": worst_fd, "fd_gamma_rel_err": err_gamma,
            "tol": tol64,
            "f32_vs_f64_gx_rel_err": float((gx32 - gx64).norm() / gx64.norm()),
            "f32_vs_f64_ggamma_rel_err": abs(gg32 - gg64) / max(abs(gg64), 1e-300)}


def vjp(args):
    import torch

    from . import synth
    from .torch import tv_iso
    noisy, clean = synth.phantom(48, 256, 256, seed=0, sigma=0.1, clean=True)
    x = torch.as_tensor(noisy.reshape(16, 3, 256, 256), device="cuda")
    c = torch.as_tensor(clean.reshape(16, 3, 256, 256), device="cuda")

    def step():
        xr = x.clone().requires_grad_(True)
        g = torch.tensor(0.1, device="cuda", requires_grad=True)
        z = tv_iso(xr, g, tol=1e-6, max_iter=5000)
        loss = ((z - c) ** 2).mean()
        loss.backward()
        return xr.grad, g.grad, loss

    step()
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    base = torch.cuda.memory_allocated()
    e0, e1 = _events()
    e0.record()
    gx, gg, loss = step()
    e1.record()
    torch.cuda.synchronize()
    t_ours = e0.elapsed_time(e1) / 1e3
    peak_ours = torch.cuda.max_memory_allocated() - base
    # 400 unrolled FISTA iterations (the dual method, autograd through every one)
    torch.cuda.reset_peak_memory_stats()
    base = torch.cuda.memory_allocated()
    e0.record()
    xr = x.clone().requires_grad_(True)
    g = torch.tensor(0.1, device="cuda", requires_grad=True)
    z = _unrolled_fista(xr, g, 400)
    loss_u = ((z - c) ** 2).mean()
    loss_u.backward()
    e1.record()
    torch.cuda.synchronize()
    t_unrolled = e0.elapsed_time(e1) / 1e3
    peak_unrolled = torch.cuda.max_memory_allocated() - base
    out = {"workload": "vjp", "metric": "forward+backward seconds, (16,3,256,256) fp32, implicit VJP",
           "value": t_ours, "unit": "s", "peak_torch_bytes": int(peak_ours),
           "unrolled400_seconds": t_unrolled, "unrolled400_peak_bytes": int(peak_unrolled),
           "loss": float(loss.detach()), "loss_unrolled400": float(loss_u.detach()), "ggamma": float(gg)}
    if not getattr(args, "no_checks", False):
        # the checks on the first sample's three channels (a float64 solve to gap
        # 1e-12 and 16 fixed-iteration solves of the differences: minutes for all 48)
        out["checks"] = vjp_checks(noisy[:3].reshape(1, 3, 256, 256), clean[:3].reshape(1, 3, 256, 256), ndir=8)
    return out


def _unrolled_fista(x, gamma, iters):
    """Plain dual FISTA for isotropic TV in torch ops (tau = 1/8), unrolled."""
    import torch
    k = 2

    def div(u):  # x - G^T u = x + (u[p] - u[p - e])
        z = x.clone()
        z = z + u[0] - torch.nn.functional.pad(u[0][..., :-1, :], (0, 0, 1, 0))
        z = z + u[1] - torch.nn.functional.pad(u[1][..., :, :-1], (1, 0, 0, 0))
        return z

    def grad(z):
        g0 = torch.nn.functional.pad(z[..., 1:, :] - z[..., :-1, :], (0, 0, 0, 1))
        g1 = torch.nn.functional.pad(z[..., :, 1:] - z[..., :, :-1], (0, 1, 0, 0))
        return torch.stack([g0, g1])

    u = torch.zeros((k,) + tuple(x.shape), device=x.device, dtype=x.dtype)
    v = u
    t = 1.0
    for _ in range(iters):
        c = v + grad(div(v)) / 8.0
        n = torch.sqrt((c * c).sum(0)).clamp_min(1e-30)
        un = c * torch.clamp(gamma / n, max=1.0)
        tn = 0.5 * (1 + math.sqrt(1 + 4 * t * t))
        v = un + (t - 1) / tn * (un - u)
        u, t = un, tn
    return div(u)


def serve(args):
    from . import serve as srv
    return srv.run(seconds=args.serve_seconds, workers=getattr(args, "serve_workers", 16))
