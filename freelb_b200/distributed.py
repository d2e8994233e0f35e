"""Blocks on several GPUs: one process per GPU, NCCL between them.

The reference runs a block-structured domain over MPI ranks with
NormalCommunicate copying each block's overlap layer from the neighbour that
owns those cells (src/data_struct/block_lattice.hh:1419-1503,
src/parallel/communicator.h).  Here each rank holds an FLB_BLOCKS_HALO handle
of the blocks it owns; the copies between its own blocks stay on the device
inside flb_step, and the copies whose source block lives on another rank are
packed into one device buffer per peer (flb_exchange_pack), moved with NCCL
point-to-point sends and receives (torch.distributed, one batch per step) and
scattered into the overlap slots (flb_exchange_unpack) before the next step.

A z-slab decomposition of a cavity is ``slabs(ni, nranks)``: each face crossed
by five directions, nx * ny cells per face.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from . import Lattice, _stream

ELEM_BYTES = {"fp32": 4, "fp16s": 2, "fp64": 8, "fp32s": 4}
HALO_MODES = {"normal": C.HALO_NORMAL, "full": C.HALO_FULL}


def slabs(ni: int, nranks: int):
    """The ni^3 cavity interior split into nranks z-slabs (one block per rank),
    in the form geometry.uneven_blocks returns."""
    if nranks < 1 or nranks > ni:
        raise ValueError(f"{nranks} slabs of {ni} planes")
    n = ni + 2
    cuts = [ni * r // nranks for r in range(nranks + 1)]
    return [{"x0": 0, "y0": 0, "z0": a, "ex": ni, "ey": ni, "ez": b - a,
             "nx": n, "ny": n, "nz": b - a + 2, "ox": 0, "oy": 0, "oz": a}
            for a, b in zip(cuts[:-1], cuts[1:])]


def _descs(blocks):
    arr = (C.BlockDesc * len(blocks))()
    for k, b in enumerate(blocks):
        arr[k].nx, arr[k].ny, arr[k].nz = int(b["nx"]), int(b["ny"]), int(b["nz"])
        arr[k].ox, arr[k].oy, arr[k].oz = int(b["ox"]), int(b["oy"]), int(b["oz"])
        arr[k].omega = 0.0
    return arr


def plan(blocks, owners, rank, halo_mode="normal"):
    """Host-only exchange plan of `rank`: {peer: (elements sent, elements received)}."""
    n = len(blocks)
    own = (ctypes.c_int * n)(*[int(o) for o in owners])
    npeers = ctypes.c_int()
    peers = (ctypes.c_int * n)()
    snd = (ctypes.c_longlong * n)()
    rcv = (ctypes.c_longlong * n)()
    C.call("flb_exchange_plan", n, _descs(blocks), own, int(rank), HALO_MODES[halo_mode], n,
           ctypes.byref(npeers), peers, snd, rcv)
    return {int(peers[j]): (int(snd[j]), int(rcv[j])) for j in range(npeers.value)}


def nccl_exchange(send, recv, group=None):
    """Move the per-peer buffers: one batch of point-to-point sends and receives
    (every rank posts its sends and receives in peer order, so the batch pairs
    up on both sides).  The operations are ordered after the work already on
    torch's current stream, and that stream waits for them (req.wait())."""
    import torch.distributed as dist
    ops = []
    for peer in sorted(set(send) | set(recv)):
        if peer in recv and recv[peer].numel():
            ops.append(dist.P2POp(dist.irecv, recv[peer], peer, group))
        if peer in send and send[peer].numel():
            ops.append(dist.P2POp(dist.isend, send[peer], peer, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


def host_exchange(send, recv, group=None):
    """The same exchange through host memory, for process groups whose backend
    moves only CPU tensors (gloo): device buffers are copied out on torch's
    current stream (which synchronises it), sent and received as one batch, and
    copied back on that stream."""
    import torch.distributed as dist
    hsend = {p: b.cpu() for p, b in send.items() if b.numel()}
    hrecv = {p: b.new_empty(b.shape, device="cpu") for p, b in recv.items() if b.numel()}
    nccl_exchange(hsend, hrecv, group)
    for p, b in hrecv.items():
        recv[p].copy_(b)


class RankLattice:
    """This rank's part of a block-decomposed lattice (the blocks it owns, in
    global order) and its per-peer exchange buffers on the current device."""

    def __init__(self, blocks, owners, rank, tau, storage="fp32", halo_mode="normal", **kw):
        import torch
        self.blocks, self.owners, self.rank = list(blocks), list(owners), int(rank)
        self.local = [b for b, o in zip(self.blocks, self.owners) if o == self.rank]
        if not self.local:
            raise ValueError(f"rank {rank} owns no block")
        tuples = [(b["nx"], b["ny"], b["nz"], b["ox"], b["oy"], b["oz"]) for b in self.local]
        self.lat = Lattice.blocks(tuples, tau, mode="halo", storage=storage, **kw)
        if halo_mode != "normal":
            self.lat.set_halo_mode(halo_mode)
        n = len(self.blocks)
        own = (ctypes.c_int * n)(*[int(o) for o in self.owners])
        h = ctypes.c_void_p()
        C.call("flb_exchange_create", self.lat._h, n, _descs(self.blocks), own, self.rank,
               ctypes.byref(h))
        self._ex = h
        npeers = ctypes.c_int()
        peers = (ctypes.c_int * n)()
        snd = (ctypes.c_longlong * n)()
        rcv = (ctypes.c_longlong * n)()
        C.call("flb_exchange_peers", h, n, ctypes.byref(npeers), peers, snd, rcv)
        eb = ELEM_BYTES[storage]
        dev = torch.device("cuda", torch.cuda.current_device())
        self.send, self.recv = {}, {}
        for j in range(npeers.value):
            p = int(peers[j])
            self.send[p] = torch.empty(int(snd[j]) * eb, dtype=torch.uint8, device=dev)
            self.recv[p] = torch.empty(int(rcv[j]) * eb, dtype=torch.uint8, device=dev)

    def pack(self, stream=None):
        for p, buf in self.send.items():
            C.call("flb_exchange_pack", self._ex, self.lat._h, p, ctypes.c_void_p(buf.data_ptr()),
                   _stream(stream))

    def unpack(self, stream=None):
        for p, buf in self.recv.items():
            C.call("flb_exchange_unpack", self._ex, self.lat._h, p,
                   ctypes.c_void_p(buf.data_ptr()), _stream(stream))

    def step(self, n=1, stream=None, exchange=None, group=None):
        """n steps: stream-collide plus local halo (flb_step), then pack, the
        exchange and unpack.  `exchange`: None or "nccl" (NCCL through
        torch.distributed), "host" (through host memory, for gloo), or a
        callable taking this RankLattice.  `stream` (a torch.cuda.Stream, a raw
        cudaStream_t as int, or None for torch's current stream) orders all of
        it: the exchange runs with that stream as torch's current stream, so
        the library's pack / unpack kernels and the transfers between them are
        ordered on one stream."""
        import torch
        if stream is None:
            ts = torch.cuda.current_stream()
        elif isinstance(stream, int):
            ts = torch.cuda.ExternalStream(stream)
        else:
            ts = stream
        move = None
        if not callable(exchange):
            move = {None: nccl_exchange, "nccl": nccl_exchange, "host": host_exchange}.get(exchange)
            if move is None:
                raise ValueError(f"unknown exchange {exchange!r}")
        with torch.cuda.stream(ts):
            for _ in range(n):
                self.lat.step(1, ts)
                self.pack(ts)
                if move is not None:
                    move(self.send, self.recv, group)
                else:
                    exchange(self)
                self.unpack(ts)

    def close(self):
        if getattr(self, "_ex", None) and self._ex.value:
            C.load().flb_exchange_destroy(self._ex)
            self._ex = ctypes.c_void_p()
        self.lat.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
