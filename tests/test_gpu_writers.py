"""GPU: .vti output of a running domain and restart from a checkpoint."""
import numpy as np
import pytest

from asl_b200 import lbgk as A
from asl_b200 import workloads as W
from asl_b200.writers import WriterVTKXML, load_checkpoint, read_vti, save_checkpoint

pytestmark = pytest.mark.gpu


def test_vti_of_running_domain(gpu, tmp_path):
    w = W.channel_cylinder(size=(32, 16, 16), radius=3.0, center=(8.0, 8.0))
    lb, bcs = W.build_lbgk(w, "f32")
    lb.run(10, bcs)
    out = WriterVTKXML(str(tmp_path / "cyl"), lb.block)
    out.addScalars("rho", lambda: lb.getRho(np.float32))
    out.addVector("velocity", lambda: lb.getVelocity(np.float32))
    d = read_vti(out.write())
    assert np.array_equal(d["rho"], lb.getRho(np.float32)[1:-1, 1:-1, 1:-1])
    assert np.array_equal(d["velocity"], lb.getVelocity(np.float32)[:, 1:-1, 1:-1, 1:-1])
    assert np.abs(d["velocity"][0]).max() > 0.01  # the flow is there
    lb.run(10, bcs)
    d1 = read_vti(out.write())
    assert (tmp_path / "cyl_1.vti").exists()
    assert not np.array_equal(d1["velocity"], d["velocity"])


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("fuse", [False, True])
def test_restart_from_checkpoint_is_bitwise(gpu, tmp_path, storage, fuse):
    w = W.channel_cylinder(size=(24, 12, 12), radius=2.5, center=(6.0, 6.0))
    ref, rbcs = W.build_lbgk(w, storage, fuse=fuse)
    ref.run(14, rbcs)
    a, abcs = W.build_lbgk(w, storage, fuse=fuse)
    a.run(7, abcs)  # odd: the checkpoint is taken in representation B
    path = save_checkpoint(a, str(tmp_path / "ck"))
    b, bbcs = W.build_lbgk(w, storage, fuse=fuse)
    assert load_checkpoint(b, path) == 7
    b.run(7, bbcs)
    assert b.steps == 14
    assert np.array_equal(b.getF(), ref.getF(), equal_nan=True)
    assert np.array_equal(b.getVelocity()[:, 1:-1, 1:-1, 1:-1], ref.getVelocity()[:, 1:-1, 1:-1, 1:-1])
    assert np.array_equal(b.getRho()[1:-1, 1:-1, 1:-1], ref.getRho()[1:-1, 1:-1, 1:-1])
    c, _ = W.build_lbgk(W.channel_cylinder(size=(16, 12, 12)), storage)
    with pytest.raises(ValueError):
        load_checkpoint(c, path)
    other = "f64" if storage != "f64" else "f32"
    d, _ = W.build_lbgk(w, other)
    with pytest.raises(A.L.ASLError):
        load_checkpoint(d, path)
