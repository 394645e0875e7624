"""x-slab decomposition of one domain over several GPUs (one process per GPU,
torch.distributed for the transport), or over several domains of one
process (for tests and single-GPU use).

A workload of Nx x Ny x Nz cells is cut into slabs of whole x planes. Each
slab is an LBGK domain of its own (not periodic in x: its two ghost planes
stand for the neighbours' boundary planes). Every step is

    stream-collide of each slab  ->  face exchange  ->  separate conditions

where the face exchange (aslb_lbgk_halo_pack / _unpack) moves, across every
interior face, the populations that cross it: after an odd step the ones the
boundary cells pushed into the ghost plane, after an even step the
boundary-plane ones the next odd step pulls in. x walls (X0 / XE conditions)
exist on the first / last slab only; an x-periodic workload closes the ring.
Conditions on y / z walls and on maps are built per slab from the slab's
part of the map (ghost planes included), so every link is handled by the
slab that owns its fluid end, as in the undivided domain.

Across processes the step overlaps the exchange with the interior
(overlapped_step): the two boundary planes are advanced first on the
domain's stream (aslb_lbgk_step_planes), packed and handed to the transport
while the interior planes run on a second stream; unpacking, then the
separate conditions, follow on the domain's stream once the interior is
joined. The exchange only touches slots of the boundary and ghost planes that
no interior cell reads or writes in the same step, so the overlap changes no
result. With NCCL the transfers are ordered on the streams (no host wait);
the host-staged transport is the same choreography for CPU process groups.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from . import _lib as L
from . import lbgk as A
from . import workloads as W


def split(nx: int, parts: int):
    """(x0, nx_r) of each slab: whole planes, sizes differing by at most one."""
    base, extra = divmod(nx, parts)
    out, x0 = [], 0
    for r in range(parts):
        n = base + (1 if r < extra else 0)
        out.append((x0, n))
        x0 += n
    return out


def slab_workload(w: W.Workload, r: int, parts: int) -> W.Workload:
    x0, n = split(w.size[0], parts)[r]
    px = w.periodic[0]
    bcs = []
    for s in w.bcs:
        walls = tuple(v for v in s.walls
                      if not ((v == "X0" and (r != 0 or px)) or (v == "XE" and (r != parts - 1 or px))))
        if s.walls and not walls:
            continue
        bcs.append(replace(s, walls=walls))
    m = None if w.map is None else np.ascontiguousarray(w.map[x0:x0 + n + 2])
    return replace(w, name="%s_slab%d" % (w.name, r), size=(n, w.size[1], w.size[2]),
                   periodic=(False, w.periodic[1], w.periodic[2]), bcs=bcs, map=m,
                   position=(w.position[0] + x0 * w.dx, w.position[1], w.position[2]))


class Slab:
    """One slab: its LBGK, its conditions, and its device face buffers."""

    def __init__(self, w: W.Workload, r: int, parts: int, storage="f32", fuse=False, **kw):
        import torch
        self.r, self.parts, self.periodic_x = r, parts, w.periodic[0]
        self.x0, self.nx = split(w.size[0], parts)[r]
        self.w = slab_workload(w, r, parts)
        self.lb, self.bcs = W.build_lbgk(self.w, storage=storage, fuse=fuse, **kw)
        nbytes = int(self.lb.lib.aslb_lbgk_halo_bytes(self.lb.h))
        self.send = [torch.empty(nbytes, dtype=torch.uint8, device="cuda") for _ in range(2)]
        self.recv = [torch.empty(nbytes, dtype=torch.uint8, device="cuda") for _ in range(2)]
        self.stream = torch.cuda.ExternalStream(self.lb.stream)
        self.side = torch.cuda.Stream()  # the interior planes of an overlapped step

    def neighbour(self, face: int):
        """Rank across `face` (0 low, 1 high), or None at a wall."""
        o = self.r + (1 if face else -1)
        if 0 <= o < self.parts:
            return o
        return o % self.parts if self.periodic_x else None

    def pack(self):
        for face in (0, 1):
            if self.neighbour(face) is not None:
                L.check(self.lb.lib.aslb_lbgk_halo_pack(self.lb.h, face, self.send[face].data_ptr()), "halo_pack")

    def unpack(self):
        for face in (0, 1):
            if self.neighbour(face) is not None:
                L.check(self.lb.lib.aslb_lbgk_halo_unpack(self.lb.h, face, self.recv[face].data_ptr()), "halo_unpack")

    def sync(self):
        self.lb.sync()


def local_exchange(slabs):
    """Face exchange among the slabs of one process."""
    for s in slabs:
        s.pack()
    for s in slabs:
        s.sync()
    for s in slabs:
        for face in (0, 1):
            o = s.neighbour(face)
            if o is not None:
                s.recv[face].copy_(slabs[o].send[1 - face])
    import torch
    torch.cuda.synchronize()
    for s in slabs:
        s.unpack()


def exchange_plan(rank: int, parts: int, periodic_x: bool):
    """Point-to-point operations of one face exchange, in posting order:
    ("send", peer, face) / ("recv", peer, face). Sends go high face first,
    receives low face first, so that with two slabs on a ring (both faces
    facing the same peer) the k-th message between a pair is matched by the
    k-th receive: my high-face data lands in the peer's low-face buffer."""
    def nb(face):
        o = rank + (1 if face else -1)
        if 0 <= o < parts:
            return o
        return o % parts if periodic_x else None

    ops = []
    for face in (1, 0):
        if nb(face) is not None:
            ops.append(("send", nb(face), face))
    for face in (0, 1):
        if nb(face) is not None:
            ops.append(("recv", nb(face), face))
    return ops


def dist_exchange(slab: Slab, group=None):
    """Face exchange of this rank's slab with its neighbours over NCCL,
    after a whole step (pack, transfers and unpack ordered on the domain's
    stream)."""
    slab.pack()
    nccl_transport(slab, group)
    slab.unpack()


def nccl_transport(slab: Slab, group=None):
    """The face buffers to and from the neighbours with NCCL point-to-point
    operations, ordered on the domain's stream: they start after the pack
    and the unpack enqueued next waits for them, without a host wait."""
    import torch
    import torch.distributed as dist
    ops = []
    with torch.cuda.stream(slab.stream):
        for kind, peer, face in exchange_plan(slab.r, slab.parts, slab.periodic_x):
            if peer == slab.r:  # a single slab on an x-periodic ring
                if kind == "send":
                    slab.recv[1 - face].copy_(slab.send[face])
                continue
            if kind == "send":
                ops.append(dist.P2POp(dist.isend, slab.send[face], peer, group))
            else:
                ops.append(dist.P2POp(dist.irecv, slab.recv[face], peer, group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


def host_transport(slab: Slab, group=None):
    """The same exchange staged through host memory, for process groups
    whose backend moves host tensors (gloo): the packed faces are copied to
    the host (waiting for the pack), sent, and the received ones copied back
    on the domain's stream."""
    import torch
    import torch.distributed as dist
    slab.stream.synchronize()
    send = [b.cpu() for b in slab.send]
    recv = [torch.empty_like(b) for b in send]
    ops = []
    for kind, peer, face in exchange_plan(slab.r, slab.parts, slab.periodic_x):
        if peer == slab.r:
            if kind == "send":
                recv[1 - face].copy_(send[face])
            continue
        if kind == "send":
            ops.append(dist.P2POp(dist.isend, send[face], peer, group))
        else:
            ops.append(dist.P2POp(dist.irecv, recv[face], peer, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    with torch.cuda.stream(slab.stream):
        for face in (0, 1):
            if slab.neighbour(face) is not None:
                slab.recv[face].copy_(recv[face])


def step_begin(slab: Slab):
    """First half of an overlapped step: the interior planes on the side
    stream, the boundary planes on the domain's stream, then the pack."""
    lib, h, nx = slab.lb.lib, slab.lb.h, slab.nx
    if nx < 3:
        slab.lb.execute(1)
    else:
        slab.side.wait_stream(slab.stream)  # the interior starts after the previous step
        L.check(lib.aslb_lbgk_step_planes(h, 2, nx - 1, slab.side.cuda_stream), "step_planes")
        L.check(lib.aslb_lbgk_step_planes(h, 1, 1, None), "step_planes")
        L.check(lib.aslb_lbgk_step_planes(h, nx, nx, None), "step_planes")
        L.check(lib.aslb_lbgk_step_commit(h), "step_commit")
    slab.pack()


def step_end(slab: Slab):
    """Second half: unpack the received faces, join the interior, then the
    separate conditions."""
    slab.unpack()
    if slab.nx >= 3:
        slab.stream.wait_stream(slab.side)
    for b in slab.bcs:
        b.execute()


def overlapped_step(slab: Slab, transport, group=None):
    """One step of this rank's slab with the face exchange overlapping the
    interior planes."""
    step_begin(slab)
    transport(slab, group)
    step_end(slab)


def local_overlapped_step(slabs):
    """The overlapped step for the slabs of one process: each receiving copy
    waits on the sending slab's stream."""
    import torch
    for s in slabs:
        step_begin(s)
    for s in slabs:
        for face in (0, 1):
            o = s.neighbour(face)
            if o is not None:
                s.stream.wait_stream(slabs[o].stream)
                with torch.cuda.stream(s.stream):
                    s.recv[face].copy_(slabs[o].send[1 - face])
    for s in slabs:
        for face in (0, 1):
            o = s.neighbour(face)
            if o is not None:  # the sender may not overwrite its buffer before the copy
                slabs[o].stream.wait_stream(s.stream)
    for s in slabs:
        step_end(s)


def step(slabs_or_slab, nsteps: int, exchange):
    """nsteps steps: stream-collide, face exchange, separate conditions."""
    slabs = slabs_or_slab if isinstance(slabs_or_slab, (list, tuple)) else [slabs_or_slab]
    for _ in range(nsteps):
        for s in slabs:
            s.lb.execute(1)
        exchange()
        for s in slabs:
            for b in s.bcs:
                b.execute()


def _main(argv=None):
    """Weak-scaled porous channel over x slabs, one per GPU:
        python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 -m asl_b200.slabs
    Each rank owns a 512 x 256 x 256 slab of an (N * 512) x 256 x 256 channel
    and exchanges its faces over NCCL every step; rank 0 prints MLUPS."""
    import argparse
    import datetime
    import json
    import os
    import torch
    import torch.distributed as dist
    ap = argparse.ArgumentParser(prog="python -m asl_b200.slabs")
    ap.add_argument("--slab", default="512,256,256")
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=4)
    a = ap.parse_args(argv)
    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    L.check(L.load().aslb_set_device(local), "set_device")
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    sx, sy, sz = (int(v) for v in a.slab.split(","))
    w = W.porous_channel(size=(sx * world, sy, sz))
    slab = Slab(w, rank, world, fuse=True, compVel=False, compRho=False)
    for _ in range(a.warmup):
        overlapped_step(slab, nccl_transport)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    st = slab.stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(a.steps):
        overlapped_step(slab, nccl_transport)
    e1.record(st)
    e1.synchronize()
    t = torch.tensor([e0.elapsed_time(e1) / 1e3], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        print(json.dumps({"slabs": world, "cells": w.cells, "steps": a.steps,
                          "mlups": w.cells * a.steps / float(t.item()) / 1e6}))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    _main()
