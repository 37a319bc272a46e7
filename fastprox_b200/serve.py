"""A device-resident request loop for TV denoising with continuous batching,
and the one-at-a-time baseline it is measured against.

Requests arrive by a Poisson process. Each is a 2D isotropic or anisotropic
denoise (50/50) of a square image of side log-uniform in [64, 2048], or with
probability 0.05 an isotropic 128^3 volume; float32 phantom + noise(0.1),
gamma log-uniform [0.02, 0.3], tol 1e-5. Images are crops of a few seeded
phantoms with per-request noise drawn on the device.

Serving (``serve_stream``):
* 2D isotropic requests join one ragged batch (fp_b200_batch_*): admitted
  into free slots as they arrive, iterating together with those already on
  the GPU, leaving as each meets its own gap; their dual state stays on the
  device for the whole solve.
* anisotropic and 3D requests of the same shape that wait together are
  stacked into one batch on the device (one call, one step per image, each
  image stopped at its own gap; the 3D volumes are all 128^3, so they batch
  whenever several wait), run on a pool of worker streams, so their kernels
  overlap with the ragged batch's.
* admission is capped by an HBM budget: a request waits while the memory its
  solve needs (its workspace, or its share of the batch arena) would exceed it.
* the batch runs a bounded number of iterations per loop pass, so arrivals
  join it within a few iterations; workspaces come from the library's memory
  pool, so per-request set-up never synchronises the device.
The baseline (``one_at_a_time``) solves the same requests in arrival order,
one fp_prox call at a time on one stream.
Latency is measured on the host from a request's arrival to its result being
ready, and reported as p50/p99 beside images/s.
"""

from __future__ import annotations

import concurrent.futures as cf
import math
import threading
import time

import numpy as np


class Request:
    __slots__ = ("i", "t", "kind", "side", "gamma", "tol", "x", "z", "done", "bytes")

    def __init__(self, i, t, kind, side, gamma):
        self.i, self.t, self.kind, self.side, self.gamma = i, t, kind, side, gamma
        self.tol = 1e-5
        self.x = self.z = None
        self.done = None
        self.bytes = 0


def make_requests(seconds, rate=200.0, seed=0):
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        if rng.uniform() < 0.05:
            kind, side = "iso3d", 128
        else:
            kind = "iso2d" if rng.uniform() < 0.5 else "aniso2d"
            side = int(round(math.exp(rng.uniform(math.log(64), math.log(2048)))))
        reqs.append(Request(len(reqs), t, kind, side, float(math.exp(rng.uniform(math.log(0.02), math.log(0.3))))))
    return reqs


class ImageSource:
    """Crops of seeded phantoms (on the device) plus per-request noise."""

    def __init__(self, seed=0):
        import torch

        from . import synth
        self.big = torch.as_tensor(synth.phantom(2, 2048, 2048, seed=seed, sigma=0.0), device="cuda")
        self.vol = torch.as_tensor(synth.phantom3d(1, 128, 128, 128, seed=seed, sigma=0.0)[0], device="cuda")
        self.gen = torch.Generator(device="cuda")
        self.gen.manual_seed(seed)

    def image(self, r):
        import torch
        if r.kind == "iso3d":
            base = self.vol
        else:
            s = r.side
            k = r.i % 2
            o = (r.i * 7919) % (2048 - s + 1)
            base = self.big[k, o:o + s, (r.i * 104729) % (2048 - s + 1):][:, :s]
        return (base + 0.1 * torch.randn(base.shape, generator=self.gen, device="cuda")).contiguous()


def _solve_one(r):
    from .image_tv import TVAniso, TVIso
    op = TVIso(3) if r.kind == "iso3d" else (TVIso(2) if r.kind == "iso2d" else TVAniso(2))
    z, info = op.solve(r.x[None], r.gamma, tol=r.tol, max_iter=5000, with_dual=False)
    return z[0], info


def solve_group(group, ops=None):
    """One call for requests of the same kind and shape: their images stacked
    into one batch on the device, one step per image (fp_prox_steps), each
    image stopped at its own gap. ops caches an operator per kind; its
    workspace is freed after the call (the memory pool makes that cheap), so
    that the device memory held is the admitted requests', whatever shapes
    have come before. Returns the results in the group's order."""
    import torch

    from .image_tv import TVAniso, TVIso
    kind = group[0].kind
    if ops is None:
        ops = {}
    op = ops.get(kind)
    if op is None:
        op = ops[kind] = TVIso(3) if kind == "iso3d" else (TVIso(2) if kind == "iso2d" else TVAniso(2))
    x = torch.stack([r.x for r in group])
    steps = torch.tensor([r.gamma for r in group], dtype=torch.float64, device=x.device)
    z, info = op.solve(x, steps, tol=group[0].tol, max_iter=5000, with_dual=False)
    op.release()
    return [z[i] for i in range(len(group))], info


class Admission:
    """HBM-budget admission: a request is admitted while the device memory
    its solve needs (its workspace, or its share of a batch arena) fits under
    the budget next to what is already admitted; it waits otherwise, and its
    bytes return to the budget when it finishes. Host-side accounting only,
    thread-safe (workers release from their threads)."""

    def __init__(self, budget_bytes, reserved=0):
        self.budget = float(budget_bytes)
        self.used = float(reserved)
        self.peak = self.used
        self._lock = threading.Lock()

    def try_admit(self, nbytes):
        with self._lock:
            if self.used + nbytes > self.budget:
                return False
            self.used += nbytes
            self.peak = max(self.peak, self.used)
            return True

    def release(self, nbytes):
        with self._lock:
            self.used -= nbytes
            if self.used < -1e-6:
                raise RuntimeError("admission released more than it admitted")


def _ws_bytes(r):
    n = r.side ** 3 if r.kind == "iso3d" else r.side * r.side
    k = 3 if r.kind == "iso3d" else 2
    return n * 4 * (3 + 5 * k) + n * 24


def serve_stream(reqs, src, budget_bytes=120e9, workers=16, steps=8, group_max=8, keep=False):
    """Continuous batching. Returns per-request latencies (s) and the span;
    with keep, each request's result stays in r.z."""
    import torch

    from .batch import RaggedBatch
    arena_px = 64 * 1024 * 1024
    main = torch.cuda.Stream()
    # worker threads use the device while the batch runs: plain launches
    batch = RaggedBatch(max_images=512, max_pixels=arena_px, graphs=False, stream=main.cuda_stream)
    arena_bytes = arena_px * 44  # d 4, u and v ping-pong 32, dual 8
    adm = Admission(budget_bytes, reserved=arena_bytes)
    streams = [torch.cuda.Stream() for _ in range(workers)]
    tls = threading.local()
    counter = iter(range(1 << 30))

    def work(group, ready):
        if not hasattr(tls, "s"):
            tls.s = streams[next(counter) % workers]
            tls.ops = {}
        tls.s.wait_event(ready)
        with torch.cuda.stream(tls.s):
            zs, _ = solve_group(group, tls.ops)
            tls.s.synchronize()
        if keep:
            for r, z in zip(group, zs):
                r.z = z
        return group

    pool = cf.ThreadPoolExecutor(workers)
    futures = {}
    inflight = {}  # batch slot -> request
    waiting = []
    lat = np.zeros(len(reqs))
    t0 = time.perf_counter()
    nxt = 0
    done = 0
    while done < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt].t <= now:
            r = reqs[nxt]
            with torch.cuda.stream(main):
                r.x = src.image(r)
            r.bytes = _ws_bytes(r)
            waiting.append(r)
            nxt += 1
        still = []
        groups = {}
        for r in waiting:
            if r.kind == "iso2d":
                slot = batch.admit(r.x, r.gamma, r.tol, max_iter=5000)
                if slot is None:
                    still.append(r)
                else:
                    inflight[slot] = r
            else:
                # anisotropic and 3D requests of one shape waiting together
                # solve as one batch (up to group_max), admitted as one
                g = groups.setdefault((r.kind, r.side), [])
                if len(g) < group_max:
                    g.append(r)
                else:
                    still.append(r)
        for g in groups.values():
            nbytes = sum(r.bytes for r in g)
            if adm.try_admit(nbytes):
                ready = torch.cuda.Event()
                ready.record(main)
                futures[pool.submit(work, g, ready)] = (g, nbytes)
            else:
                still.extend(g)
        waiting = sorted(still, key=lambda q: q.i)
        if batch.pending:
            for slot, z, gap, it, conv in batch.run(steps=steps, max_chunks=1):
                r = inflight.pop(slot)
                if keep:
                    r.z = z
                lat[r.i] = time.perf_counter() - t0 - r.t
                done += 1
        finished = [f for f in futures if f.done()]
        for f in finished:
            g, nbytes = futures.pop(f)
            f.result()
            tnow = time.perf_counter() - t0
            for r in g:
                lat[r.i] = tnow - r.t
            adm.release(nbytes)
            done += len(g)
        if not batch.pending and not finished and not (nxt < len(reqs) and reqs[nxt].t <= now):
            time.sleep(0.0005)
    span = time.perf_counter() - t0
    pool.shutdown()
    return lat, span


def one_at_a_time(reqs, src, service=None):
    """The plain path; `service` (a dict) collects the GPU seconds per kind."""
    import torch
    lat = np.zeros(len(reqs))
    t0 = time.perf_counter()
    for r in reqs:
        now = time.perf_counter() - t0
        if r.t > now:
            time.sleep(r.t - now)
        r.x = src.image(r)
        torch.cuda.synchronize()
        ts = time.perf_counter()
        _solve_one(r)
        torch.cuda.synchronize()
        te = time.perf_counter()
        if service is not None:
            service[r.kind] = service.get(r.kind, 0.0) + (te - ts)
        lat[r.i] = te - t0 - r.t
    return lat, time.perf_counter() - t0


def run(seconds=20.0, rate=200.0, seed=0, workers=16):
    import torch
    src = ImageSource(seed)
    warm = make_requests(0.2, rate, seed + 1)
    serve_stream(warm, src, workers=workers)
    reqs = make_requests(seconds, rate, seed)
    lat, span = serve_stream(reqs, src, workers=workers)
    reqs_b = make_requests(seconds, rate, seed)
    service = {}
    lat_b, span_b = one_at_a_time(reqs_b, src, service)
    torch.cuda.synchronize()
    kinds = {k: sum(r.kind == k for r in reqs) for k in ("iso2d", "aniso2d", "iso3d")}
    return {"workload": "serve", "metric": "serve p50/p99 latency (ms) and images/s, Poisson arrivals",
            "rate_per_s": rate, "seconds": seconds, "requests": len(reqs), "kinds": kinds, "workers": workers,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "images_per_s": len(reqs) / span,
            "plain_p50_ms": float(np.percentile(lat_b, 50) * 1e3), "plain_p99_ms": float(np.percentile(lat_b, 99) * 1e3),
            "plain_images_per_s": len(reqs_b) / span_b,
            "plain_service_s": {k: round(v, 3) for k, v in service.items()}}
