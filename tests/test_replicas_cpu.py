"""Multi-GPU bench path on CPU: replicas only (independent solves per rank, no data-path
collective); the job's time is the max over ranks.  Two gloo ranks stand in for GPUs."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(1.5 + rank, world)
        W = bench.workload(nmodels=2, nelx=10, nelz=5, nt=10, seed0=1000 * rank)
        out[rank] = (got, float(W["vels"].sum()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_per_rank_models():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 2.5                  # the slowest rank's time
    assert out[0][1] != out[1][1]                         # each replica solves its own models


def test_single_rank_is_identity():
    assert bench.max_over_ranks(3.25, 1) == 3.25


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    class A:
        pass
    assert bench.run_reference(A()) is None                # returns at once, no work
