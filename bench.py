"""Throughput of the image-TV prox on B200 (isotropic TV, dual FISTA stopped on
the duality gap), through libfastprox_b200's C ABI.

Workload (one step = one fp_prox_steps call over one batch): 64 float32 images
of 512 x 512, each a piecewise-constant phantom (20 rectangles and 10 disks,
intensities U[0, 1] on 0) plus N(0, 0.1^2) noise; one pixel-weight map
U[0.5, 1.5] for the batch; steps cycling through gamma = 0.05, 0.1, 0.2 over
the images; every image stopped at duality gap <= 1e-6 |x|^2 / 2. Seeded
synthetic data (no dataset is involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). ``value`` is images/s with inputs resident in
HBM; ``e2e`` the same through host (pinned) arrays, copies included;
``roofline`` the achieved HBM rate of the dominant kernel (its algorithmic
bytes per launch / its event-timed launch duration) and of the whole call
(algorithmic bytes per pixel-iteration x pixel-iterations / time) against the
measured copy bandwidth; ``cpu_baseline`` the reference C library on the host cores.
``--impl reference`` times the reference's own CPU implementation (its C
library, built from its sources into oracle/_ref) on a bounded sample.
``parity`` compares the images the CPU leg solved with the GPU's results for
the same images (relative 2-norm error, largest entry error against
1 + max|x|, iteration counts), and states the error of both against the
reference run in float64 to gap 1e-12 on one image, beside the GPU's certified
error for it.
Multi-GPU: replicas (each rank its own batch, no data-path collective);
``--gpus N`` without a launcher's environment starts the N ranks itself.
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import socket
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

B, H, W = 64, 512, 512
# DRAM bytes (read + write) of one launch of the dominant kernel, the quad
# launch (four iterations over the 64 images, the fourth with the gap check),
# from one ncu capture of this batch (profiles/iso2d_quad_64x512_fp32.md:
# 378.6 MB read + 232.7 MB written): below the 4 x 40 B per pixel of its four
# iterations, since d, u, v and alpha are read once for all four and only the
# fourth's u, v are written.
QUAD_TRAFFIC = 611245056
QUAD_KIND, QUAD_ITERS = 3, 4  # fp_b200_workspace_step_times kind of the quad launch, its iterations
GAMMAS = (0.05, 0.1, 0.2)
TOL, MAX_ITER = 1e-6, 20000
BYTES_PER_PIXEL_ITER = 40  # d 4 + u 8 + v 8 in, u 8 + v 8 out, alpha 4 (fp32)
WORKLOAD = "tv_iso 2D, 64 x 512^2 fp32 phantom+noise(0.1), pixel weights U[0.5,1.5], gamma {0.05,0.1,0.2}, gap<=1e-6"


def launch_replicas(n):
    """Re-runs this script as n ranks on one node (torch.distributed.run, one
    process per GPU, rendezvous on 127.0.0.1) with the same arguments; rank 0
    prints the line. Returns the launcher's exit status."""
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", str(n),
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(pathlib.Path(__file__).resolve()),
           *sys.argv[1:]]
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "1"))
    return subprocess.run(cmd, env=env).returncode


def reduce_max_time(t, dist, device):
    """The slowest rank's device time: the whole job's time (replicas)."""
    import torch
    tt = torch.tensor([t], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def make_inputs(seed=0):
    from fastprox_b200 import synth
    x = synth.phantom(B, H, W, seed=seed, sigma=0.1)
    alpha = synth.pixel_weights((H, W), seed=seed + 1)
    steps = np.array([GAMMAS[i % len(GAMMAS)] for i in range(B)], np.float64)
    return x, alpha, steps


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (SM clock, throttle reasons) during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
            return self

        def read():
            for line in self.proc.stdout:
                self.samples.append([f.strip() for f in line.split(",")])
        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[0]))
                mx.append(float(s[1]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, s[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference(x, alpha, steps, nimg, threads=None):
    """The reference C library (oracle/_ref) on the first nimg images: images/s."""
    from oracle import ref_capi
    threads = threads or ref_capi.default_threads()
    xs = np.ascontiguousarray(x[:nimg])
    t0 = time.perf_counter()
    r = ref_capi.solve(xs, 0.0, iso=True, k=2, spatial=alpha, tol=TOL, max_iter=MAX_ITER, threads=threads,
                       steps=steps[:nimg])
    dt = time.perf_counter() - t0
    return nimg / dt, threads, r


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref_capi
    cfg = {"workload": WORKLOAD, "global_batch": B, "image": [H, W], "dtype_in": "float32",
           "sample_images_per_step": 3}
    if not ref_capi.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference C library not built (oracle/_ref)"}))
        return
    x, alpha, steps = make_inputs()
    vals = []
    for i in range(args.warmup + args.steps):
        v, threads, _ = cpu_reference(x, alpha, steps, 3)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    line = {"metric": "TV-prox images/s at gap<=1e-6 (512^2 fp32)", "value": value, "unit": "images/s",
            "impl": "reference", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 3 / value * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "images/s", "cores": threads, "kind": "reference",
                             "sample": "3 of the 64 images per step (one per gamma), reference fp_prox_steps"},
            "e2e": {"value": value, "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _nrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def parity(x, alpha, steps, z_gpu, iters_gpu, zerr_gpu, r):
    """The GPU's results on the images the reference solved (r: the CPU
    leg's result on the first len(r.iters) images), and the error of both
    against the reference in float64 at gap 1e-12 on image 0."""
    from oracle import ref_capi
    n = len(r.iters)
    rel = [_nrel(z_gpu[i], r.z[i]) for i in range(n)]
    emax = float(np.abs(z_gpu[:n].astype(np.float64) - r.z).max() / (1 + np.abs(x[:n]).max()))
    r64 = ref_capi.solve(x[:1].astype(np.float64), float(steps[0]), iso=True, k=2, spatial=alpha, tol=1e-12,
                         max_iter=200000)
    return {"images": n, "gamma": [float(g) for g in steps[:n]], "max_rel_err": max(rel),
            "rel_err": rel, "max_entry_err": emax,
            "iters_gpu": [int(i) for i in iters_gpu[:n]], "iters_reference": [int(i) for i in r.iters],
            "iters_equal": bool(np.array_equal(iters_gpu[:n], r.iters)),
            "fp64_1e12": {"image": 0, "iters": int(r64.iters[0]), "err_gpu_f32": _nrel(z_gpu[0], r64.z[0]),
                          "err_reference_f32_input": _nrel(r.z[0], r64.z[0]), "zerr_gpu": float(zerr_gpu[0])}}


def uneven_parity(sample):
    """The uneven workload's ragged results on a seeded sample of its images
    against the reference C library on the same images (each with its own
    step and tolerance): relative 2-norm errors and iteration counts."""
    from oracle import ref_capi
    if not ref_capi.available():
        return None
    errs, its = [], []
    for i, x, gamma, tol, z, it in sample:
        r = ref_capi.solve(x[None], gamma, iso=True, k=2, tol=tol, max_iter=5000)
        errs.append(_nrel(z, r.z[0]))
        its.append((it, int(r.iters[0])))
    return {"images": [s[0] for s in sample], "max_rel_err_vs_reference": max(errs), "rel_err": errs,
            "iters_gpu_vs_reference": its}


def profile_case(kind="iso"):
    """iso: the benchmark batch (64 x 512^2, pixel weights, three steps)
    solved for exactly 12 iterations: the cold start, quad launches at
    iterations 1 and 5 (four iterations each, the fourth with the gap check),
    a pair at 9 and single steps at 11 and 12 (the check at max_iter). aniso: 16 of its
    images, anisotropic with edge weights, solved to gap 1e-6 (every kernel of
    the method, polish included). iso3d: 8 volumes of 128^3 for 8 iterations.
    ragged: 64 images of 512^2 in a ragged batch (32-row tiles, plain
    launches), gamma 0.1, gap 1e-6, at most 200 iterations."""
    import torch

    from fastprox_b200 import TVAniso, TVIso, synth
    if kind == "iso3d":
        x = torch.as_tensor(synth.phantom3d(8, 128, 128, 128, seed=0), device="cuda")
        z, info = TVIso(3).solve(x, 0.1, tol=0.0, max_iter=8, with_dual=False)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "iso3d", "iters": int(info.iters)}))
        return
    if kind == "ragged":
        from fastprox_b200.batch import RaggedBatch
        B, H, W = 64, 512, 512
        b = RaggedBatch(max_images=B, max_pixels=B * H * W + 4096, rows=32, graphs=False)
        xs = torch.as_tensor(synth.phantom(B, H, W, seed=0), device="cuda")
        for i in range(B):
            b.admit(xs[i], 0.1, 1e-6, max_iter=200)
        n = 0
        while b.pending:
            n += len(b.run(steps=4))
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "ragged", "finished": n, **b.stats()}))
        return
    if kind == "aniso":
        B = 16
        x = torch.as_tensor(synth.phantom(B, 512, 512, seed=0), device="cuda")
        beta = synth.pixel_weights((2, 512, 512), seed=1)
        st = torch.as_tensor([(0.05, 0.1, 0.2)[i % 3] for i in range(B)], device="cuda", dtype=torch.float64)
        z, info = TVAniso(2, edge_weights=beta).solve(x, st, tol=1e-6, max_iter=2000, with_dual=False)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "aniso", "iters": int(info.iters)}))
        return
    x, alpha, steps = make_inputs()
    xt = torch.as_tensor(x, device="cuda")
    st = torch.as_tensor(steps, device="cuda")
    op = TVIso(2, pixel_weights=alpha)
    z, info = op.solve(xt, st, tol=0.0, max_iter=12, with_dual=False)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": True, "iters": int(info.iters)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--profile-case", nargs="?", const="iso", default=None, choices=["iso", "aniso", "iso3d", "ragged"],
                    help="iso: one solve of the benchmark batch with 12 iterations (tol 0); aniso: 16 images "
                         "anisotropic to gap 1e-6; iso3d: 8 x 128^3 with 8 iterations; ragged: 64 x 512^2 in a "
                         "ragged batch; the cases for ncu captures")
    ap.add_argument("--workload", default="iso512", choices=["iso512", "aniso512", "iso3d", "uneven", "vjp", "serve"],
                    help="iso512 (default, the headline line); the others report the other workloads")
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-workers", type=int, default=16, help="worker streams for anisotropic and 3D requests")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case)
        return
    if args.workload != "iso512" and args.impl == "ours":
        from fastprox_b200 import workloads
        res = getattr(workloads, args.workload)(args)
        sample = res.pop("_sample", None)
        if sample is not None and not args.no_cpu:
            res["vs_reference"] = uneven_parity(sample)
        print(json.dumps(res))
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_replicas(args.gpus))
    if args.impl == "reference":
        run_reference_arm(args)
        return

    import ctypes as C

    import torch
    import torch.distributed as dist

    from fastprox_b200 import TVIso, capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)

    x, alpha, steps = make_inputs(seed=rank)
    xt = torch.as_tensor(x, device=dev)
    st = torch.as_tensor(steps, device=dev)
    out = torch.empty_like(xt)
    op = TVIso(2, pixel_weights=alpha)
    stream = torch.cuda.current_stream(dev)
    L = capi.lib()

    def device_step():
        return op.solve(xt, st, tol=TOL, max_iter=MAX_ITER, out=out, with_dual=False)[1]

    for _ in range(max(args.warmup, 3)):
        info = device_step()
    ws = op.workspace(xt)
    kl, sl = C.c_int64(), C.c_int64()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    pix_iters = 0
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            info = device_step()
            L.fp_b200_workspace_stats(ws, C.byref(kl), C.byref(sl))
            launches += kl.value
            pix_iters += int(info.image_iters.sum()) * H * W
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    t = ev0.elapsed_time(ev1) / 1e3
    if world > 1:
        t = reduce_max_time(t, dist, dev)
        dist.barrier()
    value = world * B * args.steps / t
    ms_per_step = t / args.steps * 1e3
    assert info.converged, "benchmark solve did not converge"

    # end to end through host arrays (pinned), copies in the timed region
    xh = torch.from_numpy(x).pin_memory()
    oh = torch.empty_like(xh).pin_memory()
    xn, on = xh.numpy(), oh.numpy()
    op_host = TVIso(2, pixel_weights=alpha)
    for _ in range(2):
        op_host.solve(xn, steps, tol=TOL, max_iter=MAX_ITER, out=on, with_dual=False)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        op_host.solve(xn, steps, tol=TOL, max_iter=MAX_ITER, out=on, with_dual=False)
    torch.cuda.synchronize(dev)
    te = time.perf_counter() - t0
    if world > 1:
        te = reduce_max_time(te, dist, dev)
    e2e = world * B * e2e_steps / te

    peak, peak_kind = peaks()
    achieved = BYTES_PER_PIXEL_ITER * pix_iters / args.steps / (t / args.steps) / 1e9
    z_timed = out.cpu().numpy()  # the last timed solve's output (the kernel timing below reuses out)
    # The dominant kernel alone (after the timed region): the quad launch,
    # timed by events the library puts around each step launch, with all 64
    # images live (tol 0, 24 iterations: quads at iterations 1, 5, ..., 17).
    L.fp_b200_workspace_time_steps(ws, 1)
    op.solve(xt, st, tol=0.0, max_iter=24, out=out, with_dual=False)
    L.fp_b200_workspace_time_steps(ws, 0)
    kms, kn = C.c_double(), C.c_int64()
    L.fp_b200_workspace_step_times(ws, QUAD_KIND, C.byref(kms), C.byref(kn))
    kernel_us = kms.value / max(kn.value, 1) * 1e3
    kernel_bytes = QUAD_ITERS * BYTES_PER_PIXEL_ITER * B * H * W  # four iterations over the batch
    achieved_kernel = kernel_bytes / (kernel_us * 1e-6) / 1e9 if kn.value else None
    dram = QUAD_TRAFFIC / (kernel_us * 1e-6) / 1e9 if (kn.value and QUAD_TRAFFIC) else None
    cpu = None
    par = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            from oracle import ref_capi
            if ref_capi.available():
                v, threads, r = cpu_reference(x, alpha, steps, 3)
                cpu = {"value": v, "unit": "images/s", "cores": threads, "kind": "reference",
                       "sample": "3 of the 64 images (gamma 0.05, 0.1, 0.2), reference C fp_prox_steps, "
                                 "all host threads"}
                par = parity(x, alpha, steps, z_timed, info.image_iters, info.zerr, r)
        except Exception as e:  # the baseline is reported, not required
            cpu = {"value": None, "unit": "images/s", "cores": None, "kind": "reference", "sample": f"failed: {e}"}
    if rank == 0:
        iters = info.image_iters
        line = {
            "metric": "TV-prox images/s at gap<=1e-6 (512^2 fp32)", "value": value, "unit": "images/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "global_batch": B * world, "image": [H, W], "tol": TOL,
                       "max_iter": MAX_ITER, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (d, u, v: 604 MB per batch)",
                       "iters_per_image": {"min": int(iters.min()), "median": float(np.median(iters)),
                                           "max": int(iters.max())}},
            "roofline": {"bound": "hbm", "achieved": achieved_kernel, "peak": peak, "unit": "GB/s",
                         "frac": achieved_kernel / peak if achieved_kernel else None, "peak_kind": peak_kind,
                         "kernel": "iso2d_quad_kernel (four iterations per launch, the fourth with the gap "
                                   "check; all images live)",
                         "kernel_us": kernel_us, "kernel_launches_timed": int(kn.value),
                         "algorithmic_bytes_per_launch": kernel_bytes, "bytes_per_pixel_iter": BYTES_PER_PIXEL_ITER,
                         "traffic": QUAD_TRAFFIC, "dram_achieved": dram,
                         "dram_frac": dram / peak if dram else None,
                         "achieved_whole_call": achieved, "frac_whole_call": achieved / peak},
            "cpu_baseline": cpu,
            "parity": par,
            "e2e": {"value": e2e, "unit": "images/s", "h2d_bytes_per_step": int(x.nbytes),
                    "d2h_bytes_per_step": int(x.nbytes)},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
