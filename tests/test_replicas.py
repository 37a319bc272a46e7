"""Multi-GPU is replicas only (images are independent): every rank solves
its own batch and the job's time is the slowest rank's. The host side of
that, on CPU with the gloo backend and two ranks."""

import os
import pathlib
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    out[rank] = bench.reduce_max_time(1.0 + rank, dist, torch.device("cpu"))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_with_gloo():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == out[1] == 2.0


def test_replica_inputs_differ_per_rank_but_are_seeded():
    sys.path.insert(0, str(ROOT))
    from fastprox_b200 import synth
    a0 = synth.phantom(2, 32, 32, seed=0)
    a1 = synth.phantom(2, 32, 32, seed=1)
    assert not (a0 == a1).all()
    assert (synth.phantom(2, 32, 32, seed=1) == a1).all()


def test_bench_gpus_flag_launches_the_ranks_itself():
    """bench.py --gpus 2 outside a launcher starts two ranks (rendezvous on
    127.0.0.1) and rank 0 alone prints one line, for the world of two. The
    reference arm runs on the host cores, so this needs no GPU."""
    import json
    import subprocess

    import pytest
    from oracle import ref_capi
    if not ref_capi.available():
        pytest.skip("reference library not built (make -C oracle)")
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=600, env=env, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
