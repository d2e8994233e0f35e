"""The multi-GPU bench path runs independent cavities per rank (replicas, no
collective on the data path); the only cross-rank step is the job time, the
maximum of the per-rank device times.  Exercised here with two gloo ranks on CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.5, 40.25][rank]
        q.put((rank, bench.max_over_ranks(torch, dist, ms, torch.device("cpu"))))
    finally:
        dist.destroy_process_group()


def test_job_time_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 40.25, 1: 40.25}


def test_single_rank_is_identity():
    assert bench.max_over_ranks(torch, None, 3.5, torch.device("cpu")) == 3.5
