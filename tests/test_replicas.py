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
