"""CPU tests of the x-slab decomposition's host logic: the split, the
per-slab workloads, and the face-exchange choreography over torch.distributed
with the gloo backend (world sizes 2 and 3, walled and x-periodic), each rank
sending buffers tagged with (rank, face) and checking what arrives."""
import os
import socket

import numpy as np
import pytest

from asl_b200 import slabs as SL
from asl_b200 import workloads as W


def test_split_covers_the_domain():
    for nx, parts in ((10, 3), (7, 7), (512, 8), (5, 2)):
        s = SL.split(nx, parts)
        assert s[0][0] == 0 and sum(n for _, n in s) == nx
        assert all(s[i][0] + s[i][1] == s[i + 1][0] for i in range(parts - 1))
        assert max(n for _, n in s) - min(n for _, n in s) <= 1


def test_slab_workloads_keep_x_walls_at_the_ends():
    w = W.channel_cylinder(size=(30, 16, 12), radius=3.0, center=(8.0, 8.0))
    parts = 3
    for r in range(parts):
        ws = SL.slab_workload(w, r, parts)
        walls = [v for s in ws.bcs for v in s.walls]
        assert ("X0" in walls) == (r == 0) and ("XE" in walls) == (r == parts - 1)
        x0, n = SL.split(30, parts)[r]
        assert ws.size == (n, 16, 12) and ws.periodic[0] is False
        assert np.array_equal(ws.map, w.map[x0:x0 + n + 2])
    p = W.porous_channel(size=(24, 12, 12), rmin=2.0, rmax=3.0, solid_fraction=0.2)
    for r in range(2):
        ws = SL.slab_workload(p, r, 2)
        assert ws.periodic == (False, False, False) and ws.body_force == p.body_force


def _plan_worker(rank, world, periodic, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        send = [torch.full((4,), float(rank * 10 + f)) for f in (0, 1)]
        recv = [torch.full((4,), -1.0) for _ in (0, 1)]
        ops = []
        for kind, peer, face in SL.exchange_plan(rank, world, periodic):
            if kind == "send":
                ops.append(dist.P2POp(dist.isend, send[face], peer))
            else:
                ops.append(dist.P2POp(dist.irecv, recv[face], peer))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        q.put((rank, [float(r[0]) for r in recv]))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world,periodic", [(2, False), (2, True), (3, False), (3, True)])
def test_exchange_choreography_gloo(world, periodic):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_plan_worker, args=(r, world, periodic, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        for face in (0, 1):
            o = r + (1 if face else -1)
            if not 0 <= o < world:
                if not periodic:
                    assert got[r][face] == -1.0
                    continue
                o %= world
            # the neighbour across my face packed its opposite face for me
            assert got[r][face] == o * 10 + (1 - face), (r, face, got[r])
