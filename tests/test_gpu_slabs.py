"""GPU tests of the x-slab decomposition in one process: a domain cut into
slabs (separate LBGK objects exchanging their x faces through
aslb_lbgk_halo_pack / _unpack) advances exactly like the undivided domain,
for walled and x-periodic channels, separate and fused conditions, odd and
even step counts: the populations, density and velocity of every fluid cell
are bit-identical. (Solid cells next to a slab face may differ: their
skipped slots are not exchanged, and nothing reads them.) Every process-to-process detail of the exchange is the same
code path apart from the transport (tests/test_slabs_cpu.py covers that
with gloo)."""
import numpy as np
import pytest

from asl_b200 import slabs as SL
from asl_b200 import workloads as W

pytestmark = pytest.mark.gpu


def run_both(w, parts, steps, fuse, storage="f32"):
    ref, rbcs = W.build_lbgk(w, storage=storage, fuse=fuse)
    ref.run(steps, rbcs, use_graph=False)
    ref.sync()
    slabs = [SL.Slab(w, r, parts, storage=storage, fuse=fuse) for r in range(parts)]
    SL.step(slabs, steps, lambda: SL.local_exchange(slabs))
    for s in slabs:
        s.sync()
    return ref, slabs


@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("fuse", [False, True])
@pytest.mark.parametrize("steps", [7, 8])
def test_channel_slabs_equal_undivided(gpu, parts, fuse, steps):
    w = W.channel_cylinder(size=(36, 18, 14), radius=3.5, center=(15.0, 9.0))
    ref, slabs = run_both(w, parts, steps, fuse)
    F, R, U = ref.getF(), ref.getRho(), ref.getVelocity()
    fluid = w.map > 0
    for s in slabs:
        sl = slice(s.x0 + 1, s.x0 + s.nx + 1)
        f = s.lb.getF()
        mask = fluid[sl, 1:-1, 1:-1]
        assert np.array_equal(f[:, 1:-1, 1:-1, 1:-1][:, mask], F[:, sl, 1:-1, 1:-1][:, mask])
        assert np.array_equal(s.lb.getVelocity()[:, 1:-1, 1:-1, 1:-1][:, mask], U[:, sl, 1:-1, 1:-1][:, mask])
        assert np.array_equal(s.lb.getRho()[1:-1, 1:-1, 1:-1][mask], R[sl, 1:-1, 1:-1][mask])


@pytest.mark.parametrize("parts", [1, 2, 3])
@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_periodic_porous_slabs_equal_undivided(gpu, parts, storage):
    w = W.porous_channel(size=(30, 16, 16), rmin=2.0, rmax=3.5, solid_fraction=0.25, steps=0)
    ref, slabs = run_both(w, parts, 9, True, storage)
    F = ref.getF()
    fluid = w.map > 0
    for s in slabs:
        sl = slice(s.x0 + 1, s.x0 + s.nx + 1)
        mask = fluid[sl, 1:-1, 1:-1]
        f = s.lb.getF()
        assert np.array_equal(f[:, 1:-1, 1:-1, 1:-1][:, mask], F[:, sl, 1:-1, 1:-1][:, mask])


@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("case", ["channel", "porous"])
def test_overlapped_steps_equal_undivided(gpu, parts, case):
    """The overlapped step (boundary planes first, the interior on a second
    stream while the faces move, split with aslb_lbgk_step_planes) gives the
    undivided domain's populations bit for bit on every fluid cell."""
    if case == "channel":
        w = W.channel_cylinder(size=(36, 18, 14), radius=3.5, center=(15.0, 9.0))
    else:
        w = W.porous_channel(size=(30, 16, 16), rmin=2.0, rmax=3.5, solid_fraction=0.25, steps=0)
    steps = 9
    ref, rbcs = W.build_lbgk(w, fuse=True)
    ref.run(steps, rbcs, use_graph=False)
    ref.sync()
    slabs = [SL.Slab(w, r, parts, fuse=True) for r in range(parts)]
    for _ in range(steps):
        SL.local_overlapped_step(slabs)
    for s in slabs:
        s.sync()
    F = ref.getF()
    fluid = w.map > 0
    for s in slabs:
        assert s.lb.steps == steps
        sl = slice(s.x0 + 1, s.x0 + s.nx + 1)
        mask = fluid[sl, 1:-1, 1:-1]
        f = s.lb.getF()
        assert np.array_equal(f[:, 1:-1, 1:-1, 1:-1][:, mask], F[:, sl, 1:-1, 1:-1][:, mask])


def _gloo_slab_worker(rank, world, port, steps, out):
    import os
    import torch
    import torch.distributed as dist
    from asl_b200 import _lib as L
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    L.check(L.load().aslb_set_device(0), "set_device")
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = W.porous_channel(size=(40, 16, 16), rmin=2.0, rmax=3.5, solid_fraction=0.25, steps=0)
        slab = SL.Slab(w, rank, world, fuse=True)
        for _ in range(steps):
            SL.overlapped_step(slab, SL.host_transport)
        slab.sync()
        np.save(out % rank, slab.lb.getF())
    finally:
        dist.destroy_process_group()


def test_two_processes_exchange_real_faces(gpu, tmp_path):
    """Two processes on the one GPU, each owning a slab of an x-periodic
    porous channel, exchange their packed faces through gloo (host-staged;
    the kernels of the two processes never wait on each other) with the
    overlapped step: their populations equal the undivided domain's."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    steps = 8
    out = str(tmp_path / "slab%d.npy")
    mp.start_processes(_gloo_slab_worker, args=(2, port, steps, out), nprocs=2, join=True, start_method="spawn")
    w = W.porous_channel(size=(40, 16, 16), rmin=2.0, rmax=3.5, solid_fraction=0.25, steps=0)
    ref, rbcs = W.build_lbgk(w, fuse=True)
    ref.run(steps, rbcs, use_graph=False)
    ref.sync()
    F = ref.getF()
    fluid = w.map > 0
    for r in range(2):
        x0, n = SL.split(w.size[0], 2)[r]
        f = np.load(out % r)
        sl = slice(x0 + 1, x0 + n + 1)
        mask = fluid[sl, 1:-1, 1:-1]
        assert np.array_equal(f[:, 1:-1, 1:-1, 1:-1][:, mask], F[:, sl, 1:-1, 1:-1][:, mask])
