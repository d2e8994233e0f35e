"""Blocks on several GPUs (freelb_b200.distributed, flb_exchange_*).

CPU: the exchange plans of all ranks pair up (what rank r sends to p is what p
receives from r), and the NCCL transport's batch of sends and receives
delivers every buffer to its peer (two and three gloo ranks).  GPU: the ranks
are emulated as handles in one process on one GPU (the transport becomes a
device copy between their buffers) and must reproduce the single-block cavity
bit for bit on the fluid cells."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import freelb_b200 as F
from freelb_b200 import distributed as D
from freelb_b200 import geometry as G


def layouts():
    yield "slabs2", D.slabs(12, 2), [0, 1]
    yield "slabs4", D.slabs(16, 4), [0, 1, 2, 3]
    ub = G.uneven_blocks(24, edges=(8, 16), seed=3)
    yield "uneven3", ub, [k % 3 for k in range(len(ub))]


@pytest.mark.parametrize("halo_mode", ["normal", "full"])
def test_plans_pair_up(halo_mode):
    for name, blocks, owners in layouts():
        ranks = sorted(set(owners))
        plans = {r: D.plan(blocks, owners, r, halo_mode) for r in ranks}
        for r in ranks:
            for p, (snd, rcv) in plans[r].items():
                assert p != r and snd > 0 and rcv > 0, name
                assert plans[p][r] == (rcv, snd), (name, r, p)


def test_slab_face_counts():
    ni, n = 12, 14
    plans = {r: D.plan(D.slabs(ni, 3), [0, 1, 2], r) for r in range(3)}
    face = ni * ni * 5  # owned cells of a face x the five directions crossing it
    assert plans[0] == {1: (face, face)}
    assert plans[1] == {0: (face, face), 2: (face, face)}
    full = D.plan(D.slabs(ni, 3), [0, 1, 2], 1, "full")  # all 19 populations
    assert full == {0: (ni * ni * 19,) * 2, 2: (ni * ni * 19,) * 2}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _transport_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # a ring: every rank exchanges with both neighbours, buffer sizes differ
        peers = sorted({(rank - 1) % world, (rank + 1) % world} - {rank})
        send = {p: torch.arange(10 * (rank + 1) + p, dtype=torch.uint8) + rank for p in peers}
        recv = {p: torch.zeros(10 * (p + 1) + rank, dtype=torch.uint8) for p in peers}
        D.nccl_exchange(send, recv)
        ok = all(torch.equal(recv[p], torch.arange(10 * (p + 1) + rank, dtype=torch.uint8) + p)
                 for p in peers)
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_transport_delivers_every_buffer(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_transport_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(res.values()) and len(res) == world


def emulated_ranks(blocks, owners, storage, halo_mode="normal", tau=0.55, ulid=0.1):
    """The ranks of a decomposed cavity as handles on this GPU, with their flags
    and lid velocity."""
    ni = max(b["z0"] + b["ez"] for b in blocks)
    n = ni + 2
    flags = F.cavity_flags(ni)
    real = np.float64 if storage == "fp64" else np.float32
    u = np.zeros((n ** 3, 3), dtype=real)
    u[flags == 8, 0] = real(ulid)
    ranks = []
    for r in sorted(set(owners)):
        rl = D.RankLattice(blocks, owners, r, tau, storage=storage, halo_mode=halo_mode)
        for k, b in enumerate(rl.local):
            rl.lat.upload_flags(G.slice_block(flags, n, b), block=k)
            rl.lat.upload_field("u", G.slice_block(u, n, b, comps=3), block=k)
        ranks.append(rl)
    return ranks


def emulated_step(ranks, steps):
    by_rank = {rl.rank: rl for rl in ranks}
    for _ in range(steps):
        for rl in ranks:
            rl.lat.step(1)
            rl.pack()
        for rl in ranks:
            for p, buf in rl.recv.items():
                buf.copy_(by_rank[p].send[rl.rank])
        for rl in ranks:
            rl.unpack()
    torch.cuda.synchronize()


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["fp32", "fp64", "fp16s"])
@pytest.mark.parametrize("case", ["slabs2", "slabs4", "uneven3"])
def test_emulated_ranks_equal_single_block(gpu_ok, storage, case):
    blocks, owners = next((b, o) for name, b, o in layouts() if name == case)
    ni = max(b["z0"] + b["ez"] for b in blocks)
    n = ni + 2
    steps = 25
    ranks = emulated_ranks(blocks, owners, storage)
    emulated_step(ranks, steps)
    one = F.cavity(ni, tau=0.55, storage=storage)
    one.step(steps)
    P = one.download_pops().reshape(19, n, n, n)
    flags = F.cavity_flags(ni)
    for rl in ranks:
        for k, b in enumerate(rl.local):
            pb = rl.lat.download_pops(block=k).reshape(19, b["nz"], b["ny"], b["nx"])
            fb = G.slice_block(flags, n, b).reshape(b["nz"], b["ny"], b["nx"])
            ps = P[:, b["oz"]:b["oz"] + b["nz"], b["oy"]:b["oy"] + b["ny"],
                   b["ox"]:b["ox"] + b["nx"]]
            assert np.array_equal(pb[:, fb == 2], ps[:, fb == 2]), (case, rl.rank, k)
        rl.close()


@pytest.mark.gpu
def test_emulated_ranks_full_halo_equal_multiblock(gpu_ok):
    """With NormalFullCommunicate the distributed run equals the same blocks in
    one handle on every stored cell (overlap layers included)."""
    name, blocks, owners = list(layouts())[2]
    ni = max(b["z0"] + b["ez"] for b in blocks)
    n = ni + 2
    ranks = emulated_ranks(blocks, owners, "fp32", halo_mode="full")
    emulated_step(ranks, 20)
    whole = emulated_ranks(blocks, [0] * len(blocks), "fp32", halo_mode="full")[0]
    whole.lat.step(20)
    k_of = {}
    for rl in ranks:
        for k, b in enumerate(rl.local):
            k_of[(b["ox"], b["oy"], b["oz"])] = (rl, k)
    for k, b in enumerate(blocks):
        rl, kl = k_of[(b["ox"], b["oy"], b["oz"])]
        fb = G.slice_block(F.cavity_flags(ni), n, b)
        a = rl.lat.download_pops(block=kl).reshape(19, -1)
        w = whole.lat.download_pops(block=k).reshape(19, -1)
        assert np.array_equal(a[:, fb != 1], w[:, fb != 1]), k


@pytest.mark.gpu
def test_exchange_rejects_a_handle_that_does_not_match(gpu_ok):
    blocks = D.slabs(12, 2)
    with pytest.raises(F.FlbError):  # rank 1's handle built from rank 0's block
        wrong = [b if k == 0 else blocks[0] for k, b in enumerate(blocks)]
        rl = D.RankLattice(wrong, [0, 1], 1, 0.6)
    rl = D.RankLattice(blocks, [0, 1], 0, 0.6)
    rl.lat.set_halo_mode("full")  # the plan was built for the normal halo
    with pytest.raises(F.FlbError):
        rl.pack()
    rl.close()


def _gpu_rank(rank, world, port, q, storage, steps, own_stream):
    """One process of a two-slab cavity on cuda:0: its RankLattice, stepped with
    the host transport over gloo, returns its blocks' populations."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        torch.cuda.set_device(0)
        blocks = D.slabs(12, world)
        owners = list(range(world))
        ni = 12
        n = ni + 2
        flags = F.cavity_flags(ni)
        real = np.float64 if storage == "fp64" else np.float32
        u = np.zeros((n ** 3, 3), dtype=real)
        u[flags == 8, 0] = real(0.1)
        rl = D.RankLattice(blocks, owners, rank, 0.55, storage=storage)
        for k, b in enumerate(rl.local):
            rl.lat.upload_flags(G.slice_block(flags, n, b), block=k)
            rl.lat.upload_field("u", G.slice_block(u, n, b, comps=3), block=k)
        stream = torch.cuda.Stream() if own_stream else None
        rl.step(steps, stream=stream, exchange="host")
        torch.cuda.synchronize()
        q.put((rank, [rl.lat.download_pops(block=k) for k in range(len(rl.local))]))
        rl.close()
    except Exception as e:  # reported by the parent
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["fp32", "fp16s"])
def test_two_processes_on_one_gpu_equal_single_block(gpu_ok, storage):
    """Two processes (gloo ranks) on cuda:0, each holding the RankLattice of one
    z-slab of a 12^3 cavity, exchange their packed halo buffers through host
    memory every step; rank 1 orders its work on a stream of its own.  The
    fluid cells of both slabs equal the single-block run bit for bit.  No
    kernel of one process waits on the other's: each step's buffers cross on
    the host between the two processes' launches."""
    world, steps = 2, 20
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_rank, args=(r, world, port, q, storage, steps, r == 1))
             for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ni = 12
    n = ni + 2
    one = F.cavity(ni, tau=0.55, storage=storage)
    one.step(steps)
    P = one.download_pops().reshape(19, n, n, n)
    flags = F.cavity_flags(ni)
    for r, b in enumerate(D.slabs(ni, world)):
        assert not isinstance(res[r], str), res[r]
        pb = res[r][0].reshape(19, b["nz"], b["ny"], b["nx"])
        fb = G.slice_block(flags, n, b).reshape(b["nz"], b["ny"], b["nx"])
        ps = P[:, b["oz"]:b["oz"] + b["nz"], b["oy"]:b["oy"] + b["ny"], b["ox"]:b["ox"] + b["nx"]]
        assert np.array_equal(pb[:, fb == 2], ps[:, fb == 2]), r
