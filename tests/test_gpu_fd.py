"""GPU: FD advection-diffusion (aslb_fd_*) against the numpy oracle, coupled
to the device velocity field of a running LBGK."""
import numpy as np
import pytest

from asl_b200 import fd as FD
from asl_b200 import lbgk as A
from asl_b200 import workloads as W
from oracle.fd_oracle import fd_step

pytestmark = pytest.mark.gpu


def blob(g, dtype):
    x, y, z = np.meshgrid(*[np.arange(n, dtype=float) for n in g], indexing="ij")
    c = 0.2 + np.exp(-((x - g[0] / 3) ** 2 + (y - g[1] / 2) ** 2 + (z - g[2] / 2) ** 2) / 6.0)
    return c.astype(dtype)


@pytest.mark.parametrize("q", [7, 15, 19])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-14), (np.float32, 2e-6)])
def test_pure_diffusion_matches_oracle(gpu, q, dtype, tol):
    c = blob((14, 11, 9), dtype)
    fd = FD.generateFDAdvectionDiffusion(c, 0.12, None, q)
    ref = c.copy()
    for n in (1, 4):
        fd.execute(n)
        for _ in range(n):
            ref = fd_step(ref, 0.12, q)
        got = fd.getC()
        assert got.dtype == dtype
        assert np.abs(got - ref).max() <= tol


@pytest.mark.parametrize("q", [7, 19])
@pytest.mark.parametrize("cc", [False, True])
@pytest.mark.parametrize("storage,dtype,tol", [("f64", np.float64, 1e-13), ("f32", np.float32, 5e-6)])
def test_coupled_to_lbgk_velocity(gpu, q, cc, storage, dtype, tol):
    """The FD step reads the flow's device velocity on the domain's stream,
    after every LBGK step; the oracle gets the same velocity from the host."""
    w = W.channel_cylinder(size=(30, 14, 12), radius=2.5, center=(9.0, 7.0), u_in=0.04)
    lb, bcs = W.build_lbgk(w, storage)
    c = blob(tuple(s + 2 for s in w.size), dtype)
    fd = FD.generateFDAdvectionDiffusion(c, 0.05, lb, q, compressibilityCorrection=cc)
    FD.generateBCConstantValue(fd, 1.0, [A.X0])
    ref = fd.getC()
    assert np.all(ref[0, 1:-1, 1:-1] == 1.0)
    for _ in range(6):
        lb.run(1, bcs)
        fd.execute()
        u = lb.getVelocity(dtype)
        ref = fd_step(ref, 0.05, q, u, cc)
    got = fd.getC()
    assert np.abs(got - ref).max() <= tol
    assert np.abs(u[0]).max() > 0.01  # the flow moved


def test_unbind_on_domain_destroy_and_errors(gpu):
    w = W.channel_cylinder(size=(16, 8, 8), radius=2.0, center=(5.0, 4.0))
    lb, bcs = W.build_lbgk(w, "f32")
    c = blob((18, 10, 10), np.float32)
    with pytest.raises(A.L.ASLError):
        FD.generateFDAdvectionDiffusion(c.astype(np.float64), 0.1, lb, 7)  # FP64 field, FP32 velocity
    with pytest.raises(A.L.ASLError):
        FD.generateFDAdvectionDiffusion(blob((12, 10, 10), np.float32), 0.1, lb, 7)  # other size
    with pytest.raises(A.L.ASLError):
        FD.generateFDAdvectionDiffusion(c, 0.1, None, 27)
    fd = FD.generateFDAdvectionDiffusion(c, 0.1, lb, 7)
    lb.run(2, bcs)
    fd.execute(2)
    lb.close()
    fd.execute(1)  # unbound: pure diffusion on the FD's own stream
    ref = fd_step(fd_step(fd_step(c, 0.1, 7), 0.1, 7), 0.1, 7)
    got = fd.getC()
    assert np.isfinite(got).all() and got.shape == c.shape
    assert np.abs(got - ref).max() > 0  # the first two steps saw the flow


@pytest.mark.parametrize("q", [7, 19])
@pytest.mark.parametrize("kind", ["value", "gradient"])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-13), (np.float32, 5e-6)])
def test_map_conditions_match_oracle(gpu, q, kind, dtype, tol):
    """FD steps coupled to the cylinder flow, each followed by a value or
    normal-gradient condition on the cylinder map (the multicomponent-flow
    pattern: lbgk step, FD step, executeAll(bc))."""
    from oracle.fd_oracle import fd_map_bc
    w = W.channel_cylinder(size=(20, 12, 10), radius=2.5, center=(7.0, 6.0), u_in=0.04)
    storage = "f64" if dtype == np.float64 else "f32"
    lb, bcs = W.build_lbgk(w, storage)
    c = blob(tuple(s + 2 for s in w.size), dtype)
    fd = FD.generateFDAdvectionDiffusion(c, 0.05, lb, q)
    if kind == "value":
        fb = FD.generateBCConstantValue(fd, 0.3, w.map)
    else:
        fb = FD.generateBCConstantGradient(fd, 0.02, w.map)
    assert fb.cells > 0
    ref = fd.getC()
    for _ in range(4):
        lb.run(1, bcs)
        fd.execute()
        fb.execute()
        u = lb.getVelocity(dtype)
        ref = fd_map_bc(fd_step(ref, 0.05, q, u), w.map, q, kind == "gradient", 0.02 if kind == "gradient" else 0.3)
    assert np.abs(fd.getC() - ref).max() <= tol


@pytest.mark.parametrize("q", [7, 19])
@pytest.mark.parametrize("with_flow", [False, True])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-13), (np.float32, 5e-6)])
def test_electric_field_term_matches_oracle(gpu, q, with_flow, dtype, tol):
    """setElectricFieldParameters(phi, k, f2, q): each step subtracts
    divAgradB(c q / k, phi), alone or after the advection terms."""
    w = W.channel_cylinder(size=(18, 12, 10), radius=2.5, center=(6.0, 6.0), u_in=0.04)
    g = tuple(s + 2 for s in w.size)
    x, y, z = np.meshgrid(*[np.arange(n, dtype=float) for n in g], indexing="ij")
    phi = (0.02 * np.sin(x / 3.0) + 0.01 * np.cos(y / 2.0) * z / g[2]).astype(dtype)
    kk = (1.0 + 0.2 * np.cos(z / 2.5)).astype(dtype)
    qq = (0.5 + 0.1 * np.sin(x * y / 20.0)).astype(dtype)
    c = blob(g, dtype)
    if with_flow:
        lb, bcs = W.build_lbgk(w, "f64" if dtype == np.float64 else "f32")
        fd = FD.generateFDAdvectionDiffusion(c, 0.05, lb, q)
    else:
        lb, bcs = None, []
        fd = FD.generateFDAdvectionDiffusion(c, 0.05, None, q)
    fd.setElectricFieldParameters(phi, kk, None, qq)
    ref = fd.getC()
    for _ in range(4):
        u = None
        if lb is not None:
            lb.run(1, bcs)
            u = lb.getVelocity(dtype)
        fd.execute()
        ref = fd_step(ref, 0.05, q, u, False, electric=(phi, kk, qq))
    got = fd.getC()
    assert np.abs(got - ref).max() <= tol
    plain = fd_step(fd_step(c, 0.05, q), 0.05, q)
    assert np.abs(ref - plain).max() > 1e-5  # the term acts


@pytest.mark.parametrize("q", [15, 19])
@pytest.mark.parametrize("cc", [False, True])
def test_register_blocked_runs_across_tiles_match_oracle(gpu, q, cc):
    """FP32 d3q15 / d3q19 on a grid with more plane-tile units than resident
    blocks (each block walks a run of planes that crosses into the next
    tile, restarting its ring there), partial tiles in y and z."""
    w = W.channel_cylinder(size=(200, 20, 70), radius=4.0, center=(40.0, 10.0), u_in=0.04)
    lb, bcs = W.build_lbgk(w, "f32")
    c = blob(tuple(s + 2 for s in w.size), np.float32)
    fd = FD.generateFDAdvectionDiffusion(c, 0.05, lb, q, compressibilityCorrection=cc)
    FD.generateBCConstantValue(fd, 1.0, [A.X0])
    ref = fd.getC()
    for _ in range(3):
        lb.run(1, bcs)
        fd.execute()
        ref = fd_step(ref, 0.05, q, lb.getVelocity(np.float32), cc)
    assert np.abs(fd.getC() - ref).max() <= 5e-6
