"""GPU parity: the CUDA path (through libaslb.so's C ABI) against the CPU oracle.

Tolerances: FP64 storage must match the FP64 oracle to 1e-12 (rounding
only); FP32 storage the FP32 oracle to 1e-5 absolute on populations of order 1
over a few steps (the GPU evaluates the collision in another order, opposite
pairs and weight classes, with fused multiply-adds: tens of ulp after 7
steps); the canonical cylinder
channel to relative L2 <= 1e-4 on rho and u over interior fluid cells and
<= 1e-4 on the drag after 1000 steps.
"""
import numpy as np
import pytest

from asl_b200 import lbgk as A
from asl_b200 import workloads as W

pytestmark = pytest.mark.gpu

I4 = (slice(None), slice(1, -1), slice(1, -1), slice(1, -1))
WALLS = {"X0": 1, "XE": 2, "Y0": 4, "YE": 8, "Z0": 16, "ZE": 32}
SLICE = {"noslip": 0, "velocity": 1, "pressure": 2, "pressure_velocity": 3}
MAPK = {"noslip": 10, "velocity": 11, "pressure_velocity": 13}
VT = {15: A.d3q15(), 19: A.d3q19(), 27: A.d3q27()}


def smooth_field(g, seed, amp=0.04):
    rng = np.random.default_rng(seed)
    x = np.stack(np.meshgrid(*[np.arange(n) for n in g], indexing="ij")).astype(float)
    u = np.zeros((3, *g))
    for d in range(3):
        k = rng.integers(1, 3, size=3)
        ph = rng.uniform(0, 2 * np.pi, 3)
        u[d] = amp * np.sin(2 * np.pi * k[0] * x[0] / g[0] + ph[0]) * np.cos(2 * np.pi * k[1] * x[1] / g[1] + ph[1]) \
            * np.cos(2 * np.pi * k[2] * x[2] / g[2] + ph[2])
    rho = 1.0 + 0.01 * np.sin(2 * np.pi * x[0] / g[0])
    return rho, u


def sphere_map(g, center, r):
    pos = np.stack(np.meshgrid(*[np.arange(n) - 1.0 for n in g], indexing="ij"))
    d = np.sqrt(((pos - np.asarray(center, float).reshape(3, 1, 1, 1)) ** 2).sum(0)) - r
    return np.clip(d / 1.8, -1, 1).astype(np.float32)


@pytest.mark.parametrize("q", [15, 19, 27])
@pytest.mark.parametrize("closure", [0, 1, 2])
@pytest.mark.parametrize("storage,prec,tol", [("f64", 8, 1e-12), ("f32", 4, 1e-5)])
def test_periodic_steps_match_oracle(gpu, oracle_mod, q, closure, storage, prec, tol):
    size = (10, 9, 8)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 100 + q + closure)
    nu = 0.02
    lb = A.LBGK(A.Block(size), nu, VT[q], storage=storage, periodic=(True, True, True), body_force=(1e-3, -5e-4, 2e-4))
    lb.setClosure(closure, 0.3)
    A.LBGKUtilities(lb).initF(rho, u)
    o = oracle_mod.Oracle(size, q, prec, nu, flags=8 | 16 | 32)
    o.set_closure(closure, 0.3)
    o.set_body_force((1e-3, -5e-4, 2e-4))
    o.init_f_fields(rho, u)
    for nsteps in (1, 6):  # odd and even step counts: both AA representations
        lb.execute(nsteps)
        o.step(nsteps)
        assert np.abs(lb.getF()[I4] - o.get_f()[I4]).max() < tol
        assert np.abs(lb.getVelocity()[I4] - o.get_u()[I4]).max() < tol
        assert np.abs(lb.getRho()[1:-1, 1:-1, 1:-1] - o.get_rho()[1:-1, 1:-1, 1:-1]).max() < tol


def test_coriolis_incompressible_match_oracle(gpu, oracle_mod):
    size = (8, 7, 9)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 5)
    lb = A.LBGK(A.Block(size), 0.05, A.d3q19(), storage="f64", periodic=(True, True, True))
    lb.setCompressible(False)
    lb.setOmega((0.01, -0.02, 0.03))
    A.LBGKUtilities(lb).initF(rho, u)
    o = oracle_mod.Oracle(size, 19, 8, 0.05, flags=4 | 8 | 16 | 32)
    o.set_omega((0.01, -0.02, 0.03))
    o.init_f_fields(rho, u)
    lb.execute(5)
    o.step(5)
    assert np.abs(lb.getF()[I4] - o.get_f()[I4]).max() < 1e-12


@pytest.mark.parametrize("compressible", [False, True])
@pytest.mark.parametrize("storage,prec,tol", [("f64", 8, 1e-12), ("f32", 4, 1e-5)])
def test_coriolis_match_oracle_fp32_and_fp64(gpu, oracle_mod, compressible, storage, prec, tol):
    """The rotating-frame term with the compressible and the incompressible
    (He-Luo) equilibrium, in both storage precisions: FP64 to 1e-12, FP32 to
    1e-5 on populations of order 1 after odd and even step counts."""
    size = (9, 8, 10)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 11 + compressible)
    lb = A.LBGK(A.Block(size), 0.04, A.d3q19(), storage=storage, periodic=(True, True, True),
                body_force=(2e-4, 0.0, -1e-4))
    lb.setCompressible(compressible)
    lb.setOmega((0.012, -0.02, 0.025))
    A.LBGKUtilities(lb).initF(rho, u)
    o = oracle_mod.Oracle(size, 19, prec, 0.04, flags=(0 if compressible else 4) | 8 | 16 | 32)
    o.set_omega((0.012, -0.02, 0.025))
    o.set_body_force((2e-4, 0.0, -1e-4))
    o.init_f_fields(rho, u)
    for nsteps in (3, 4):
        lb.execute(nsteps)
        o.step(nsteps)
        assert np.abs(lb.getF()[I4] - o.get_f()[I4]).max() < tol
        assert np.abs(lb.getVelocity()[I4] - o.get_u()[I4]).max() < tol


@pytest.mark.parametrize("closure", ["asl_intent", "smagorinsky", "learned"])
def test_fp16_storage_with_closures_against_fp64_oracle(gpu, oracle_mod, closure):
    """FP16 shifted storage with each closure against the FP64 oracle (the
    learned closure as a network whose output is the constant Cs^2 = 0.3^2,
    which is Smagorinsky with Cs = 0.3): the velocity stays within 2e-4 of
    the oracle's (|u| ~ 0.04) over 40 steps of a decaying periodic field."""
    from asl_b200 import _lib as L
    from asl_b200 import closure as CL
    from oracle import mlp_oracle as M
    size = (20, 18, 16)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 31)
    nu = 0.01
    lb = A.LBGK(A.Block(size), nu, A.d3q19(), storage="f16", periodic=(True, True, True))
    o = oracle_mod.Oracle(size, 19, 8, nu, flags=8 | 16 | 32)
    if closure == "asl_intent":
        lb.setClosure(L.CLOSURE_ASL_INTENT)
        o.set_closure(1)
    elif closure == "smagorinsky":
        lb.setClosure(L.CLOSURE_SMAGORINSKY, 0.3)
        o.set_closure(2, 0.3)
    else:
        p = np.zeros(M.param_count(), dtype=np.float32)
        p[-1] = np.log(np.expm1(0.3 ** 2 / CL.OUT_SCALE))
        lb.setMLP(CL.pack(p, np.concatenate([np.zeros(9), np.ones(9)]).astype(np.float32)))
        lb.setClosure(L.CLOSURE_MLP)
        lb.setMLPPeriod(4)
        o.set_closure(2, 0.3)
    A.LBGKUtilities(lb).initF(rho, u)
    o.init_f_fields(rho, u)
    lb.execute(40)
    o.step(40)
    err = np.abs(lb.getVelocity()[I4] - o.get_u()[I4]).max()
    assert err < 2e-4, err
    assert np.abs(lb.getRho()[1:-1, 1:-1, 1:-1] - o.get_rho()[1:-1, 1:-1, 1:-1]).max() < 2e-4


@pytest.mark.slow
def test_porous_channel_1000_steps_fp32_matches_oracle(gpu, oracle_mod):
    """A reduced porous channel (96x48x48, seeded spheres, periodic x, body
    force, no-slip walls and spheres fused into the stream-collide kernel) for
    1000 steps in FP32 against the FP32 oracle (separate conditions): relative
    L2 of u over the fluid cells <= 1e-4, permeability within 1e-4. The body
    force is 2e-4 (velocities of order 1e-2): two FP32 evaluations in
    different orders differ by about 1e-7 on populations of order 1, which is
    a relative 1e-3 of the velocity at the benchmark's g = 1e-6."""
    w = W.porous_channel(size=(96, 48, 48), rmin=3.0, rmax=7.0, g=2e-4, steps=1000)
    lb, bcs = W.build_lbgk(w, storage="f32", compVel=False, compRho=False, fuse=True)
    o = oracle_mod.Oracle(w.size, 19, 4, w.nu, flags=8)
    o.set_body_force(w.body_force)
    o.init_f(1.0, (0, 0, 0))
    ids = [o.bc_slice(0, 4 | 8 | 16 | 32), o.bc_map(10, w.map)]
    lb.run(w.steps - 1, bcs, use_graph=True)
    lb.requestMacro()
    lb.run(1, bcs)
    for _ in range(w.steps):
        o.step(1)
        for i in ids:
            o.bc_execute(i)
    fluid = w.map[1:-1, 1:-1, 1:-1] > 0
    ug = lb.getVelocity()[I4][:, fluid]
    uo = o.get_u()[I4][:, fluid]
    assert np.linalg.norm(ug - uo) / np.linalg.norm(uo) <= 1e-4
    kg, ko = ug[0].sum() / fluid.size, uo[0].sum() / fluid.size
    assert abs(kg - ko) <= 1e-4 * abs(ko)


@pytest.mark.parametrize("q", [15, 19, 27])
@pytest.mark.parametrize("storage,prec,tol", [("f64", 8, 1e-12), ("f32", 4, 2e-5)])
def test_boundaries_and_force_match_oracle(gpu, oracle_mod, q, storage, prec, tol):
    size = (11, 9, 10)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 40 + q, amp=0.02)
    sphere = sphere_map(g, (4.0, 3.5, 4.0), 2.2)
    vmap = sphere_map(g, (8.5, 5.0, 6.0), 1.5)
    plan = [("slice", "velocity", ("X0",), 0.0, (0.03, 0.01, 0.0)),
            ("slice", "pressure", ("XE",), 1.01, (0, 0, 0)),
            ("slice", "noslip", ("Y0", "YE"), 0.0, (0, 0, 0)),
            ("slice", "pressure_velocity", ("Z0", "ZE"), 0.99, (0.01, 0.0, -0.02)),
            ("map", "noslip", sphere, 0.0, (0, 0, 0)),
            ("map", "velocity", vmap, 0.0, (0.0, 0.02, 0.01)),
            ("map", "pressure_velocity", vmap, 1.02, (0.01, 0.0, 0.0))]
    lb = A.LBGK(A.Block(size), 0.03, VT[q], storage=storage)
    A.LBGKUtilities(lb).initF(rho, u)
    o = oracle_mod.Oracle(size, q, prec, 0.03)
    o.init_f_fields(rho, u)
    bcs, ids = [], []
    for kind, name, where, p, uu in plan:
        if kind == "slice":
            walls = [getattr(A, w) for w in where]
            bcs.append({"noslip": lambda: A.generateBCNoSlip(lb, walls),
                        "velocity": lambda: A.generateBCConstantVelocity(lb, uu, walls),
                        "pressure": lambda: A.generateBCConstantPressure(lb, p, walls),
                        "pressure_velocity": lambda: A.generateBCConstantPressureVelocity(lb, p, uu, walls)}[name]())
            ids.append(o.bc_slice(SLICE[name], sum(WALLS[w] for w in where), p, uu))
        else:
            bcs.append({"noslip": lambda: A.generateBCNoSlip(lb, where),
                        "velocity": lambda: A.generateBCVelocity(lb, A.generatePFConstant(uu), where),
                        "pressure_velocity": lambda: A.generateBCConstantPressureVelocity(lb, p, uu, where)}[name]())
            ids.append(o.bc_map(MAPK[name], where, p, uu))
    force = A.generateComputeSurfaceForce(lb, sphere)
    for step in range(5):
        lb.execute()
        o.step(1)
        A.executeAll(bcs)
        for bid in ids:
            o.bc_execute(bid)
        got, fld = force.execute(r0=(4.0, 3.5, 4.0), field=True)
        want, wfld = o.force(sphere, r0=(4.0, 3.5, 4.0), field=True)
        assert np.abs(got - want).max() < 50 * tol * max(1.0, np.abs(want).max())
        assert np.abs(fld - wfld).max() < 10 * tol + 1e-6
        assert np.abs(lb.getF()[I4] - o.get_f()[I4]).max() < tol


def test_rotation_velocity_map_matches_oracle(gpu, oracle_mod):
    size = (12, 12, 6)
    g = tuple(s + 2 for s in size)
    cyl = np.clip((np.sqrt((np.arange(g[0])[:, None, None] - 1 - 5.5) ** 2 + (np.arange(g[1])[None, :, None] - 1 - 5.5) ** 2
                           + 0 * np.arange(g[2])[None, None, :]) - 2.5) / 1.8, -1, 1).astype(np.float32)
    lb = A.LBGK(A.Block(size), 0.05, A.d3q19(), storage="f64", periodic=(False, False, True))
    A.LBGKUtilities(lb).initF((0.0, 0.0, 0.0))
    bc = [A.generateBCNoSlip(lb, [A.X0, A.XE, A.Y0, A.YE]),
          A.generateBCVelocity(lb, A.generatePFRotationField((0, 0, 0.01), (5.5, 5.5, 0.0)), cyl)]
    o = oracle_mod.Oracle(size, 19, 8, 0.05, flags=32)
    o.init_f(1.0, (0, 0, 0))
    ids = [o.bc_slice(0, 1 | 2 | 4 | 8), o.bc_map(12, cyl, omega=(0, 0, 0.01), center=(5.5, 5.5, 0.0))]
    for _ in range(8):
        lb.execute()
        A.executeAll(bc)
        o.step(1)
        for i in ids:
            o.bc_execute(i)
    assert np.abs(lb.getF()[I4] - o.get_f()[I4]).max() < 1e-12


def test_graph_run_bitwise_equals_eager(gpu):
    w = W.channel_cylinder(size=(40, 24, 20), radius=4.0, center=(12.0, 12.0), steps=0)
    a, abcs = W.build_lbgk(w)
    b, bbcs = W.build_lbgk(w)
    a.run(37, abcs, use_graph=False)
    b.run(37, bbcs, use_graph=True)
    assert np.array_equal(a.getF(np.float32)[I4], b.getF(np.float32)[I4])
    assert np.array_equal(a.getVelocity(np.float32), b.getVelocity(np.float32))


def test_checkpoint_roundtrip(gpu):
    w = W.channel_cylinder(size=(24, 16, 12), radius=3.0, center=(8.0, 8.0), steps=0)
    a, abcs = W.build_lbgk(w, storage="f64")
    a.run(11, abcs, use_graph=False)
    f = a.getF()
    b, bbcs = W.build_lbgk(w, storage="f64")
    b.setF(f)
    a.run(6, abcs, use_graph=False)
    b.run(6, bbcs, use_graph=False)
    assert np.array_equal(a.getF()[I4], b.getF()[I4])


def test_mass_reduction_known_answers(gpu):
    # test/testMath/testReductionFunction.cc:37-67 known answers, through the
    # FP64 device reduction: 101 cells of density 2 sum to 202, 100001 cells
    # of density 6 sum to 600006 (sum of weights is 1 to rounding).
    for size, rho, want in [((101, 1, 1), 2.0, 202.0), ((11, 9091, 1), 6.0, 600006.0)]:
        lb = A.LBGK(A.Block(size), 0.1, A.d3q19(), storage="f64", periodic=(True, True, True))
        A.LBGKUtilities(lb).initF(rho, (0.0, 0.0, 0.0))
        mom = lb.moments()
        assert abs(mom[0] - want) <= 1e-13 * want
        assert np.abs(mom[1:]).max() < 1e-12


def test_mass_conservation_closed_box_fp64(gpu):
    size = (20, 18, 16)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 9, amp=0.03)
    lb = A.LBGK(A.Block(size), 0.02, A.d3q19(), storage="f64")
    A.LBGKUtilities(lb).initF(rho, u)
    bc = [A.generateBCNoSlip(lb, [A.X0, A.XE, A.Y0, A.YE, A.Z0, A.ZE])]
    A.executeAll(bc)
    m0 = lb.moments()[0]
    lb.run(200, bc)
    assert abs(lb.moments()[0] - m0) < 1e-11 * m0


def test_fp16_storage_error_bound(gpu, oracle_mod):
    # FP16 shifted storage with FP32 arithmetic against the FP64 oracle on a
    # decaying periodic field: velocity error stays below 1e-4 (|u| ~ 0.04).
    size = (24, 20, 16)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 77)
    lb = A.LBGK(A.Block(size), 0.02, A.d3q19(), storage="f16", periodic=(True, True, True))
    A.LBGKUtilities(lb).initF(rho, u)
    o = oracle_mod.Oracle(size, 19, 8, 0.02, flags=8 | 16 | 32)
    o.init_f_fields(rho, u)
    lb.execute(50)
    o.step(50)
    err = np.abs(lb.getVelocity()[I4] - o.get_u()[I4]).max()
    assert err < 1e-4, err


def test_errors_raise(gpu):
    with pytest.raises(A.L.ASLError):
        A.LBGK(A.Block((4, 4, 4)), -1.0, A.d3q19())
    lb = A.LBGK(A.Block((4, 4, 4)), 0.1, A.d3q19(), periodic=(True, False, False))
    with pytest.raises(A.L.ASLError):
        A.generateBCNoSlip(lb, [A.X0])  # wall on a periodic axis
    with pytest.raises(A.L.ASLError):
        lb.setClosure(3)  # learned closure without a network
    with pytest.raises(A.L.ASLError):
        A.generateBCNoSlip(lb, np.ones((3, 3, 3), np.float32))  # map of the wrong shape


@pytest.mark.slow
def test_channel_cylinder_parity_1000_steps(gpu, cylinder_oracle):
    """The canonical cylinder channel (128x64x64, D3Q19, FP32, 1000 steps)
    against the FP32 oracle: relative L2 of rho and u over interior fluid
    cells <= 1e-4, drag within 1e-4 relative."""
    w = cylinder_oracle["workload"]
    lb, bcs = W.build_lbgk(w, storage="f32")
    lb.run(w.steps, bcs)
    fluid = w.map[1:-1, 1:-1, 1:-1] > 0
    r_g, r_o = lb.getRho()[1:-1, 1:-1, 1:-1][fluid], cylinder_oracle["rho"][1:-1, 1:-1, 1:-1][fluid]
    u_g = lb.getVelocity()[I4][:, fluid]
    u_o = cylinder_oracle["u"][I4][:, fluid]
    assert np.linalg.norm(r_g - r_o) / np.linalg.norm(r_o) <= 1e-4
    assert np.linalg.norm(u_g - u_o) / np.linalg.norm(u_o) <= 1e-4
    force = A.generateComputeSurfaceForce(lb, w.map)
    got = force.execute(r0=(32.0, 32.0, 31.5))
    want = cylinder_oracle["force"]
    assert abs(got[0] - want[0]) <= 1e-4 * abs(want[0])


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("case", ["porous", "cylinder"])
def test_fused_noslip_bitwise_equals_separate_condition(gpu, storage, case):
    """Folding the no-slip conditions (walls and map) into the stream-collide
    kernel leaves every population (solid and ghost cells included), the
    density, velocity, mass and surface force bit-identical."""
    if case == "porous":
        w = W.porous_channel(size=(64, 32, 32), rmin=2.0, rmax=5.0, solid_fraction=0.35, steps=0)
    else:
        w = W.channel_cylinder(size=(48, 24, 20), radius=5.0, center=(14.0, 12.0), steps=0)
    a, abcs = W.build_lbgk(w, storage=storage)
    b, bbcs = W.build_lbgk(w, storage=storage, fuse=True)
    assert bbcs[-1].fused and bbcs[-2].fused and not abcs[-1].fused
    assert sum(x.kernels for x in bbcs) < sum(x.kernels for x in abcs)
    for n in (13, 12):
        a.run(n, abcs)
        b.run(n, bbcs)
        assert np.array_equal(a.getF(), b.getF(), equal_nan=True)
        assert np.array_equal(a.getVelocity(), b.getVelocity())
        assert np.array_equal(a.getRho(), b.getRho())
        assert np.array_equal(a.moments(), b.moments())
        fa = A.generateComputeSurfaceForce(a, w.map).execute(r0=(1.0, 2.0, 3.0))
        fb = A.generateComputeSurfaceForce(b, w.map).execute(r0=(1.0, 2.0, 3.0))
        assert np.array_equal(fa, fb)


@pytest.mark.parametrize("fuse", ["none", "walls", "map", "both"])
@pytest.mark.parametrize("variant", [0, 1, 2])
def test_unnormalised_map_matches_oracle(gpu, oracle_mod, fuse, variant):
    """A raw (unnormalised) distance map leaves solid cells below the -0.9999
    guard next to fluid; those links are not bounce-back and stream collided
    solid populations, with or without fusing, exactly as in the oracle."""
    size = (20, 14, 12)
    g = tuple(s + 2 for s in size)
    pos = np.stack(np.meshgrid(*[np.arange(n) - 1.0 for n in g], indexing="ij"))
    raw = (np.sqrt(((pos - np.array([8.0, 6.5, 5.5]).reshape(3, 1, 1, 1)) ** 2).sum(0)) - 3.5).astype(np.float32)
    lb = A.LBGK(A.Block(size), 0.05, A.d3q19(), storage="f64")
    lb.setKernel(variant)
    A.LBGKUtilities(lb).initF((0.02, 0.0, 0.0))
    bcs = [A.generateBCConstantVelocity(lb, (0.02, 0, 0), [A.X0]), A.generateBCConstantPressure(lb, 1.0, [A.XE]),
           A.generateBCNoSlip(lb, [A.Y0, A.YE, A.Z0, A.ZE]), A.generateBCNoSlip(lb, raw)]
    if fuse in ("walls", "both"):
        bcs[2].fuse()
    if fuse in ("map", "both"):
        bcs[3].fuse()
    if fuse == "walls":
        bcs = bcs[:2] + [bcs[3], bcs[2]]  # fused conditions go last (both no-slip: order-free)
    o = oracle_mod.Oracle(size, 19, 8, 0.05)
    o.init_f(1.0, (0.02, 0, 0))
    ids = [o.bc_slice(1, 1, 0, (0.02, 0, 0)), o.bc_slice(2, 2, 1.0), o.bc_slice(0, 4 | 8 | 16 | 32), o.bc_map(10, raw)]
    for n in range(1, 16):
        lb.run(1, bcs)
        o.step(1)
        for i in ids:
            o.bc_execute(i)
        err = np.abs(lb.getF()[I4] - o.get_f()[I4]).max()
        assert err < 1e-12, (n, err)


def test_fused_condition_must_come_last(gpu):
    w = W.channel_cylinder(size=(24, 16, 12), radius=3.0, center=(8.0, 8.0), steps=0)
    lb, bcs = W.build_lbgk(w)
    bcs[-1].fuse()
    with pytest.raises(A.L.ASLError):
        lb.run(4, [bcs[-1]] + bcs[:-1])


def test_destroy_domain_before_its_conditions(gpu):
    """Destroying a domain detaches its conditions and force objects, which
    may then be destroyed in any order (Python's collector picks one)."""
    w = W.channel_cylinder(size=(24, 16, 12), radius=3.0, center=(8.0, 8.0), steps=0)
    lb, bcs = W.build_lbgk(w)
    force = A.generateComputeSurfaceForce(lb, w.map)
    lb.run(3, bcs)
    lb.close()
    with pytest.raises(A.L.ASLError):
        bcs[0].execute()
    with pytest.raises(A.L.ASLError):
        force.execute()
    del bcs, force


@pytest.mark.parametrize("q", [15, 19, 27])
@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("shape,periodic", [((6, 5, 300), (True, True, True)),    # two z segments, z wrap
                                            ((9, 7, 40), (False, True, True)),    # 4 rows per tile, partial group
                                            ((5, 3, 17), (True, False, False)),   # short rows
                                            ((4, 3, 192), (False, True, False)),  # rows of 192: 256-cell segments
                                            ((4, 5, 96), (True, False, True))])   # rows of 96, z wrap
def test_kernel_variants_bitwise_equal(gpu, q, storage, shape, periodic):
    g = tuple(s + 2 for s in shape)
    rho, u = smooth_field(g, 3 + q)
    lbs = []
    for variant in (0, 1, 2):
        lb = A.LBGK(A.Block(shape), 0.03, VT[q], storage=storage, periodic=periodic, body_force=(1e-4, 0, 0))
        lb.setKernel(variant)
        A.LBGKUtilities(lb).initF(rho, u)
        walls = [w for a, w in ((0, (A.X0, A.XE)), (1, (A.Y0, A.YE)), (2, (A.Z0, A.ZE))) if not periodic[a] for w in w]
        bcs = [A.generateBCNoSlip(lb, walls)] if walls else []
        lbs.append((lb, bcs))
    for lb, bcs in lbs:
        lb.run(7, bcs)
        lb.sync()
    assert [lb.kernel for lb, _ in lbs] == [0, 1, 2]
    for lb, _ in lbs[1:]:
        assert np.array_equal(lbs[0][0].getF(), lb.getF(), equal_nan=True)
        assert np.array_equal(lbs[0][0].getVelocity(), lb.getVelocity())


@pytest.mark.parametrize("nz", [33, 40, 65, 70, 100])
@pytest.mark.parametrize("periodic", [(True, True, True), (False, True, True), (True, False, False)])
def test_periodic_faces_bitwise_across_kernels(gpu, nz, periodic):
    """Cells on periodic faces go to the face kernel; the two-cells-per-thread
    kernel also leaves it the z partners of the pairs it skips (z = 33, and
    nz - 32 when nz is the second cell of its pair). Every cell must still be
    advanced exactly once: the pair kernel (variant 0, fused FP32), the
    one-cell kernel (variant 2) and the TMA kernel (variant 1) agree bit for
    bit, with fused walls on the non-periodic axes and a fused sphere map."""
    shape = (12, 10, nz)
    g = tuple(s + 2 for s in shape)
    rho, u = smooth_field(g, nz)
    m = sphere_map(g, (6.0, 4.5, nz / 2.0), 3.5)
    out = []
    for variant in (0, 1, 2):
        lb = A.LBGK(A.Block(shape), 0.04, A.d3q19(), periodic=periodic, body_force=(2e-4, 1e-4, -1e-4))
        lb.setKernel(variant)
        A.LBGKUtilities(lb).initF(rho, u)
        walls = [w for a, w in ((0, (A.X0, A.XE)), (1, (A.Y0, A.YE)), (2, (A.Z0, A.ZE))) if not periodic[a] for w in w]
        bcs = ([A.generateBCNoSlip(lb, walls)] if walls else []) + [A.generateBCNoSlip(lb, m)]
        for b in bcs:
            b.fuse()
        lb.run(9, bcs)
        lb.sync()
        out.append((lb.getF(), lb.getVelocity()))
    for f, v in out[1:]:
        assert np.array_equal(out[0][0], f, equal_nan=True)
        assert np.array_equal(out[0][1], v)


def test_kernel_variants_fused_porous_bitwise(gpu):
    w = W.porous_channel(size=(80, 40, 36), rmin=2.0, rmax=5.0, solid_fraction=0.35, steps=0)
    out = []
    for variant in (0, 1, 2):
        lb, bcs = W.build_lbgk(w, fuse=True)
        lb.setKernel(variant)
        lb.run(9, bcs)
        lb.sync()
        out.append(lb.getF())
    for o in out[1:]:
        assert np.array_equal(out[0], o, equal_nan=True)


@pytest.mark.parametrize("storage,prec,tol", [("f64", 8, 1e-11), ("f32", 4, 1e-4)])
def test_vehicle_d3q27_downscale_matches_oracle(gpu, oracle_mod, storage, prec, tol):
    """The D3Q27 vehicle tunnel (velocity inlet, far field and moving floor,
    pressure outlet, fused no-slip obstacles) on a small grid against the
    oracle: rho and u over interior fluid cells (FP64: absolute 1e-11; FP32:
    relative L2 1e-4) and the drag / lift of the obstacles."""
    w = W.vehicle_d3q27(size=(64, 32, 32), steps=40)
    lb, bcs = W.build_lbgk(w, storage=storage, fuse=True)
    o = oracle_mod.Oracle(w.size, 27, prec, w.nu)
    o.init_f(1.0, w.init_u)
    ids = []
    for s in w.bcs:
        if s.kind == "map_noslip":
            ids.append(o.bc_map(10, w.map))
        else:
            ids.append(o.bc_slice(W.SLICE_KIND[s.kind], sum(W.WALL_BITS[x] for x in s.walls), s.p, s.u))
    lb.run(w.steps, bcs)
    for _ in range(w.steps):
        o.step(1)
        for i in ids:
            o.bc_execute(i)
    fluid = w.map[1:-1, 1:-1, 1:-1] > 0
    r_g, r_o = lb.getRho()[1:-1, 1:-1, 1:-1][fluid], o.get_rho()[1:-1, 1:-1, 1:-1][fluid]
    u_g, u_o = lb.getVelocity()[I4][:, fluid], o.get_u()[I4][:, fluid]
    if storage == "f64":
        assert np.abs(r_g - r_o).max() <= tol
        assert np.abs(u_g - u_o).max() <= tol
    else:
        assert np.linalg.norm(r_g - r_o) / np.linalg.norm(r_o) <= tol
        assert np.linalg.norm(u_g - u_o) / np.linalg.norm(u_o) <= tol
    got = A.generateComputeSurfaceForce(lb, w.map).execute()
    want = o.force(w.map, r0=(0.0, 0.0, 0.0))
    for a in (0, 2):  # drag, lift
        assert abs(got[a] - want[a]) <= (1e-9 if storage == "f64" else 1e-3) * max(abs(want[a]), 1e-6)


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("variant", [0, 2])
def test_packed_rows_bitwise_equal_aligned_rows(gpu, storage, variant):
    """The packed-row layout gives the same populations, rho and u as the
    aligned one (cylinder channel: velocity, pressure, fused walls and map)."""
    w = W.channel_cylinder(size=(40, 24, 20), radius=4.0, center=(10.0, 12.0))
    out = []
    for packed in (False, True):
        lb, bcs = W.build_lbgk(w, storage=storage, fuse=True, packed_rows=packed)
        lb.setKernel(variant)
        lb.run(11, bcs)
        lb.sync()
        out.append((lb.getF(), lb.getVelocity(), lb.getRho()))
    for a, b in zip(*out):
        assert np.array_equal(a, b, equal_nan=True)


def test_packed_rows_reject_tma_variant(gpu):
    lb = A.LBGK(A.Block((8, 8, 8)), 0.02, A.d3q19(), packed_rows=True)
    with pytest.raises(A.L.ASLError):
        lb.setKernel(1)


def test_fused_cells_with_both_link_kinds(gpu):
    """Map A is solid for x <= 5, map B (inside A) for x <= 5 and y <= 3: the
    cells x = 5, y >= 4 are skipped writers (anchors) for A and bounce-back
    readers (fluid ends) for B, so the one-word mask cannot hold them; fused
    and separate conditions still agree bit for bit."""
    size = (16, 10, 12)
    g = tuple(s + 2 for s in size)
    pos = np.stack(np.meshgrid(*[np.arange(n) - 1.0 for n in g], indexing="ij"))
    map_a = np.clip((pos[0] - 5.5) / 1.8, -1, 1).astype(np.float32)
    map_b = np.clip(np.maximum(pos[0] - 5.5, pos[1] - 3.5) / 1.8, -1, 1).astype(np.float32)
    out = []
    for fuse, variant in ((False, 0), (True, 0), (True, 2)):
        lb = A.LBGK(A.Block(size), 0.02, A.d3q19(), periodic=(False, True, True))
        lb.setKernel(variant)
        rho, u = smooth_field(g, 31)
        A.LBGKUtilities(lb).initF(rho, u)
        bcs = [A.generateBCNoSlip(lb, [A.X0, A.XE]), A.generateBCNoSlip(lb, map_a), A.generateBCNoSlip(lb, map_b)]
        if fuse:
            for b in bcs:
                b.fuse()
        lb.run(9, bcs)
        lb.sync()
        out.append(lb.getF())
    assert np.array_equal(out[0], out[1], equal_nan=True)
    assert np.array_equal(out[0], out[2], equal_nan=True)


@pytest.mark.parametrize("kind", [14, 15])
@pytest.mark.parametrize("storage,prec,tol", [("f64", 8, 1e-12), ("f32", 4, 1e-5)])
def test_deposition_and_flux_match_oracle(gpu, oracle_mod, kind, storage, prec, tol):
    """Deposition on a sphere map inside a closed box, after odd and even step
    counts: populations against the oracle, then the surface flux field and
    total (ComputeSurfaceFlux) on the same map. beta = 0.03 keeps the kinetics
    limited condition contracting (1 - beta / ((1 + lF) coef) > -1 for the
    smallest coef = 1/36); larger values make it amplify rounding step by step."""
    size = (14, 10, 12)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 70 + kind, amp=0.02)
    sphere = sphere_map(g, (6.5, 4.5, 5.5), 2.6)
    lb = A.LBGK(A.Block(size), 0.04, A.d3q19(), storage=storage)
    A.LBGKUtilities(lb).initF(rho, u)
    if kind == 14:
        dep = A.generateBCTransportLimitedDeposition(lb, 0.97, 0.4, sphere)
    else:
        dep = A.generateBCKineticsLimitedDeposition(lb, 0.97, 0.4, 0.03, sphere)
    bcs = [A.generateBCNoSlip(lb, [A.X0, A.XE, A.Y0, A.YE, A.Z0, A.ZE]), dep]
    flux = A.generateComputeSurfaceFlux(lb, sphere)
    o = oracle_mod.Oracle(size, 19, prec, 0.04)
    o.init_f_fields(rho, u)
    ids = [o.bc_slice(0, 63), o.bc_deposition(kind, sphere, 0.97, 0.4, 0.03)]
    for n in (5, 6):
        lb.run(n, bcs)
        for _ in range(n):
            o.step(1)
            for i in ids:
                o.bc_execute(i)
        assert np.abs(lb.getF()[I4] - o.get_f()[I4]).max() <= tol
        fld, tot = flux.execute()
        ofld, otot = o.flux(sphere)
        assert np.abs(fld - ofld).max() <= max(tol, 1e-6) * 10
        assert abs(tot - otot) <= max(tol, 1e-9) * 100 * max(1.0, abs(otot))
        assert np.abs(ofld).max() > 1e-4


@pytest.mark.parametrize("fuse", [False, True])
def test_flux_of_no_slip_map(gpu, oracle_mod, fuse):
    """The flux through a no-slip surface is zero link by link once the
    condition has run; with the condition fused into the stream-collide
    kernel the flux object must see the same (its links carry none)."""
    w = W.channel_cylinder(size=(32, 16, 16), radius=3.0, center=(10.0, 8.0))
    lb, bcs = W.build_lbgk(w, "f64", fuse=fuse)
    lb.run(9, bcs)
    fld, tot = A.generateComputeSurfaceFlux(lb, w.map).execute()
    assert np.abs(fld).max() <= 1e-15 and abs(tot) <= 1e-13


def test_deposition_f16_close_to_f32(gpu):
    size = (14, 10, 12)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 90, amp=0.02)
    sphere = sphere_map(g, (6.5, 4.5, 5.5), 2.6)
    out = []
    for storage in ("f32", "f16"):
        lb = A.LBGK(A.Block(size), 0.04, A.d3q19(), storage=storage)
        A.LBGKUtilities(lb).initF(rho, u)
        bcs = [A.generateBCNoSlip(lb, [A.X0, A.XE, A.Y0, A.YE, A.Z0, A.ZE]),
               A.generateBCTransportLimitedDeposition(lb, 0.97, 0.4, sphere)]
        lb.run(20, bcs)
        out.append((lb.getF()[I4], A.generateComputeSurfaceFlux(lb, sphere).execute()[1]))
    assert np.abs(out[0][0] - out[1][0]).max() <= 2e-3
    assert abs(out[0][1] - out[1][1]) <= 2e-3 * max(1.0, abs(out[0][1]))


@pytest.mark.parametrize("field", ["constant", "rotation"])
def test_velocity_map_with_computational_domain(gpu, oracle_mod, field):
    """generateBCVelocity(nm, v, map, computationalDomain) against the oracle:
    only neighbours inside the computational domain are fluid ends."""
    size = (16, 12, 10)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 41, amp=0.02)
    vmap = sphere_map(g, (7.5, 5.5, 4.5), 2.4)
    pos = np.stack(np.meshgrid(*[np.arange(n) - 1.0 for n in g], indexing="ij"))
    cd = np.where(pos[0] + 0.5 * pos[1] < 11.0, 1.0, -0.5).astype(np.float32)
    lb = A.LBGK(A.Block(size), 0.03, A.d3q19(), storage="f64")
    A.LBGKUtilities(lb).initF(rho, u)
    if field == "constant":
        v = A.generatePFConstant((0.01, 0.02, -0.01))
        kw = dict(u=(0.01, 0.02, -0.01))
        kind = MAPK["velocity"]
    else:
        v = A.generatePFRotationField((0.0, 0.0, 0.01), (7.5, 5.5, 4.5))
        kw = dict(omega=(0.0, 0.0, 0.01), center=(7.5, 5.5, 4.5))
        kind = 12
    bcs = [A.generateBCNoSlip(lb, [A.X0, A.XE, A.Y0, A.YE, A.Z0, A.ZE]), A.generateBCVelocity(lb, v, vmap, cd)]
    full = A.generateBCVelocity(lb, v, vmap)
    assert 0 < bcs[1].num_links < full.num_links
    o = oracle_mod.Oracle(size, 19, 8, 0.03)
    o.init_f_fields(rho, u)
    ids = [o.bc_slice(0, 63), o.bc_map(kind, vmap, 0.0, cdomain=cd, **kw)]
    for n in (3, 4):
        lb.run(n, bcs)
        for _ in range(n):
            o.step(1)
            for i in ids:
                o.bc_execute(i)
        assert np.abs(lb.getF()[I4] - o.get_f()[I4]).max() <= 1e-12


@pytest.mark.parametrize("kind", [20, 21, 22, 23])
@pytest.mark.parametrize("storage,prec,tol", [("f64", 8, 1e-12), ("f32", 4, 1e-5)])
def test_output_field_conditions_match_oracle(gpu, oracle_mod, kind, storage, prec, tol):
    """generateBCNoSlipVel / NoSlipRho / VelocityVel on the density and
    velocity outputs after each step, behind a fused no-slip map (field
    conditions may follow fused ones: they touch no population)."""
    size = (16, 12, 10)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 60 + kind, amp=0.02)
    m = sphere_map(g, (7.5, 5.5, 4.5), 2.4)
    lb = A.LBGK(A.Block(size), 0.03, A.d3q19(), storage=storage)
    A.LBGKUtilities(lb).initF(rho, u)
    nos = A.generateBCNoSlip(lb, m)
    walls = A.generateBCNoSlip(lb, [A.X0, A.XE, A.Y0, A.YE, A.Z0, A.ZE])
    kw = {}
    if kind == 20:
        fb = A.generateBCNoSlipVel(lb, m)
    elif kind == 21:
        fb = A.generateBCNoSlipRho(lb, m)
    elif kind == 22:
        fb = A.generateBCVelocityVel(lb, A.generatePFConstant((0.01, -0.02, 0.03)), m)
        kw = dict(u=(0.01, -0.02, 0.03))
    else:
        fb = A.generateBCVelocityVel(lb, A.generatePFRotationField((0.0, 0.02, 0.01), (7.5, 5.5, 4.5)), m)
        kw = dict(omega=(0.0, 0.02, 0.01), center=(7.5, 5.5, 4.5))
    nos.fuse()
    bcs = [walls, nos, fb]
    o = oracle_mod.Oracle(size, 19, prec, 0.03)
    o.init_f_fields(rho, u)
    ids = [o.bc_slice(0, 63), o.bc_map(10, m), o.bc_field(kind, m, **kw)]
    for n in (3, 4):
        lb.run(n, bcs)
        for _ in range(n):
            o.step(1)
            for i in ids:
                o.bc_execute(i)
        guard = (m <= 0) & (m > -0.9999)
        assert np.abs(lb.getRho()[guard] - o.get_rho()[guard]).max() <= tol
        assert np.abs(lb.getVelocity()[:, guard] - o.get_u()[:, guard]).max() <= tol
        inner = np.zeros(g, dtype=bool)
        inner[1:-1, 1:-1, 1:-1] = True
        assert np.abs(lb.getVelocity()[:, inner] - o.get_u()[:, inner]).max() <= tol


def test_output_field_conditions_reject_d3q27(gpu):
    lb = A.LBGK(A.Block((8, 8, 8)), 0.03, A.d3q27())
    m = np.ones((10, 10, 10), dtype=np.float32)
    with pytest.raises(A.L.ASLError, match="d3q27"):
        A.generateBCNoSlipVel(lb, m)


@pytest.mark.parametrize("storage,tol", [("f64", 1e-12), ("f32", 1e-5)])
def test_watchdog(gpu, storage, tol):
    """aslb_lbgk_watchdog: largest |u| and smallest rho from the populations
    agree with the velocity / density outputs (periodic box, no force: the
    collision keeps both moments); a non-finite cell is counted, not folded
    into the extremes."""
    size = (12, 10, 8)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 77, amp=0.05)
    lb = A.LBGK(A.Block(size), 0.03, A.d3q19(), storage=storage, periodic=(True, True, True))
    A.LBGKUtilities(lb).initF(rho, u)
    lb.run(5)
    wd = lb.watchdog()
    uo = lb.getVelocity()[I4]
    ro = lb.getRho()[1:-1, 1:-1, 1:-1]
    assert wd["nonfinite"] == 0
    assert abs(wd["max_u"] - np.sqrt((uo ** 2).sum(0)).max()) <= tol
    assert abs(wd["min_rho"] - ro.min()) <= tol
    f = lb.getF()
    f[3, 5, 5, 5] = np.nan
    lb.setF(f)
    wd2 = lb.watchdog()
    assert wd2["nonfinite"] == 1 and np.isfinite(wd2["max_u"]) and np.isfinite(wd2["min_rho"])


@pytest.mark.parametrize("storage,tol", [("f64", 1e-13), ("f32", 2e-6), ("f16", 2e-6)])
def test_compute_rho_velocity_from_populations(gpu, storage, tol):
    """LBGKUtilities::computeRho / computeVelocity / computeRhoVelocity:
    density and velocity of every interior cell from the populations as they
    stand, equal to the moments of the exported populations."""
    size = (10, 9, 12)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 21)
    lb = A.LBGK(A.Block(size), 0.03, A.d3q19(), storage=storage, periodic=(True, True, True), compVel=False,
                compRho=False, body_force=(1e-4, 0, 0))
    A.LBGKUtilities(lb).initF(rho, u)
    lb.execute(5)
    c, w = A.lattice_vectors(19), A.lattice_weights(19)
    f = lb.getF().astype(np.float64)
    r = np.tensordot(w, f, axes=1)
    m = np.tensordot((w[:, None] * c).T, f, axes=1)
    util = A.LBGKUtilities(lb)
    util.computeRho()
    assert np.abs(lb.getRho()[1:-1, 1:-1, 1:-1] - r[1:-1, 1:-1, 1:-1]).max() < tol
    util.computeVelocity()
    assert np.abs(lb.getVelocity()[I4] - (m / r)[I4]).max() < tol
    lb2 = A.LBGK(A.Block(size), 0.03, A.d3q19(), storage=storage, periodic=(True, True, True), compVel=False,
                 compRho=False, body_force=(1e-4, 0, 0))
    A.LBGKUtilities(lb2).initF(rho, u)
    lb2.execute(5)
    A.LBGKUtilities(lb2).computeRhoVelocity()
    assert np.array_equal(lb2.getVelocity(), lb.getVelocity()) and np.array_equal(lb2.getRho(), lb.getRho())


def test_bind_velocity_writes_the_callers_field(gpu):
    """LBGK(DataD v, ...): the domain writes its velocity into a device field
    the caller owns; unbinding returns to the domain's own field."""
    import ctypes as C
    import torch
    from asl_b200 import _lib as L
    size = (12, 10, 8)
    g = tuple(s + 2 for s in size)
    rho, u = smooth_field(g, 3)
    a = A.LBGK(A.Block(size), 0.05, A.d3q19(), periodic=(True, True, True))
    b = A.LBGK(A.Block(size), 0.05, A.d3q19(), periodic=(True, True, True))
    field = torch.zeros(3 * int(np.prod(g)), dtype=torch.float32, device="cuda")
    L.check(gpu.aslb_lbgk_bind_velocity(b.h, C.c_void_p(field.data_ptr())), "bind")
    for lb in (a, b):
        A.LBGKUtilities(lb).initF(rho, u)
        lb.run(4, use_graph=True)
        lb.sync()
    torch.cuda.synchronize()
    mine = field.cpu().numpy().reshape(3, *g)
    assert np.array_equal(mine[I4], a.getVelocity()[I4])
    assert np.array_equal(b.getVelocity()[I4], a.getVelocity()[I4])
    L.check(gpu.aslb_lbgk_bind_velocity(b.h, None), "unbind")
    b.execute(1)
    b.sync()
    assert np.array_equal(field.cpu().numpy().reshape(3, *g), mine)  # no longer written
