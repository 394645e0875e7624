"""GPU tests of batched domains (aslb_batch_*): a batch of domains of
different sizes, viscosities, obstacles and inlet velocities, stepped by one
launch per step, must give bit-identical populations to stepping every domain
on its own (the same collision and link arithmetic runs on each cell)."""
import numpy as np
import pytest

from asl_b200 import lbgk as A
from asl_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small_batch(n, seed):
    ws = W.batch_channels(n=n, steps=0, seed=seed)
    for w in ws:  # shrink to test size, keeping the seeded geometry's proportions
        assert w.q == 19
    return ws


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("fuse", [True, False])
@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_bitwise_equals_separate_domains(gpu, storage, fuse, use_graph):
    ws = small_batch(4, seed=11)
    steps = 9
    batch, lbs, bcs = W.build_batch(ws, storage=storage, fuse=fuse)
    batch.run(steps, bcs, use_graph=use_graph)
    batch.sync()
    for w, lb in zip(ws, lbs):  # references in the aligned-row layout
        ref, rbcs = W.build_lbgk(w, storage=storage, compVel=False, compRho=False, fuse=fuse)
        ref.run(steps, rbcs)
        ref.sync()
        assert lb.steps == steps
        assert np.array_equal(lb.getF(), ref.getF(), equal_nan=True), w.name


def test_batch_continues_after_single_domain_steps(gpu):
    """Parity and graph state stay consistent when batched and single-domain
    steps alternate, and the batch output (rho, u on request) matches."""
    ws = small_batch(3, seed=5)
    batch, lbs, bcs = W.build_batch(ws, fuse=True)
    refs = [W.build_lbgk(w, compVel=False, compRho=False, fuse=True) for w in ws]
    batch.run(4, bcs)
    for lb, bc in zip(lbs, bcs):
        lb.run(3, bc)
    for lb in lbs:
        lb.requestMacro()
    batch.run(6, bcs)
    batch.sync()
    for (ref, rbc) in refs:
        ref.run(7, rbc)
        ref.requestMacro()
        ref.run(6, rbc)
        ref.sync()
    for lb, (ref, _) in zip(lbs, refs):
        assert lb.steps == 13
        assert np.array_equal(lb.getF(), ref.getF(), equal_nan=True)
        assert np.array_equal(lb.getVelocity(), ref.getVelocity(), equal_nan=True)


def test_batch_rejects_mismatched_domains(gpu):
    ws = small_batch(2, seed=3)
    batch, lbs, bcs = W.build_batch(ws)
    lbs[0].execute(1)  # parities now differ
    with pytest.raises(A.L.ASLError):
        batch.run(2, bcs)
    lbs[1].execute(1)
    lbs[1].setBodyForce((1e-6, 0.0, 0.0))
    with pytest.raises(A.L.ASLError):
        batch.run(2, bcs)
    lbs[1].setBodyForce((0.0, 0.0, 0.0))
    batch.run(2, bcs)
    with pytest.raises(A.L.ASLError):
        batch.run(2, [bcs[1], bcs[0]])  # conditions of another domain
    lbs[1].close()
    with pytest.raises(A.L.ASLError):
        batch.run(2, bcs)


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_batch_launch_shapes_identical_and_tuned(gpu, storage):
    """Every launch shape (one cell per thread at 4 / 3 / 2 blocks per SM, two
    cells per thread at 3 / 2) gives the same populations; the tuner times
    them all and keeps the fastest."""
    ws = small_batch(3, seed=17)
    out = []
    for shape in (0, 1, 2, 3, 4):
        batch, lbs, bcs = W.build_batch(ws, storage=storage)
        batch.setShape(shape)
        batch.run(6, bcs)
        batch.sync()
        assert batch.shape == shape and batch.shape_times == []
        out.append([lb.getF() for lb in lbs])
    for other in out[1:]:
        for a, b in zip(out[0], other):
            assert np.array_equal(a, b, equal_nan=True)
    batch, lbs, bcs = W.build_batch(ws, storage=storage)
    batch.run(14, bcs)  # long enough for the tuner: a first step, then 2 steps per shape
    batch.sync()
    t = batch.shape_times
    assert len(t) == 5 and batch.shape == int(np.argmin(t))
    for lb in lbs:
        assert lb.steps == 14


def test_batch_runs_across_domains_bitwise(gpu):
    """More tiles than resident blocks: every group of blocks walks a run of
    planes crossing domain boundaries, its blocks interleaving the planes.
    Every launch shape gives the populations of the domains stepped alone."""
    ws = small_batch(12, seed=23)
    steps = 6
    refs = []
    for w in ws:
        ref, rbcs = W.build_lbgk(w, storage="f32", compVel=False, compRho=False, fuse=True)
        ref.run(steps, rbcs)
        ref.sync()
        refs.append(ref.getF())
    for shape in (0, 1, 2, 3, 4):
        batch, lbs, bcs = W.build_batch(ws, storage="f32")
        batch.setShape(shape)
        batch.run(steps, bcs)
        batch.sync()
        assert batch.tiles > 4 * 148  # more tiles than blocks at every residency of a B200
        for w, lb, ref in zip(ws, lbs, refs):
            assert np.array_equal(lb.getF(), ref, equal_nan=True), (shape, w.name)
