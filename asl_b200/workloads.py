"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset is involved: every geometry and initial field below is
generated from a seed (base seed 20261203, configuration k uses seed + k).

  channel_cylinder  D3Q19 128x64x64 channel, cylinder r=8 along z at (32, 32),
                    inlet u=0.05 at X0, pressure 1 at XE, no-slip Y/Z walls,
                    nu=0.01 (tau=0.53), rest start.
  porous_channel    D3Q19 512x256x256, non-overlapping random spheres
                    (r ~ U[4,12], solid fraction 0.4), periodic in x, no-slip
                    Y/Z walls, body force g=1e-6 along x, tau=0.6.
  batch_channels    256 independent D3Q19 channels, sizes x ~ U[32,128],
                    y, z ~ U[32,64] (about 47 M cells in all), each with one box
                    or sphere obstacle, inlet velocity ~ U[0.02,0.08] at X0,
                    pressure 1 at XE, no-slip Y/Z walls, tau ~ U[0.52,0.8].
  vehicle_d3q27     D3Q27 768x384x384 wind tunnel, 12 seeded boxes / vertical
                    cylinders standing on the floor (Z0), velocity 0.05 along x
                    at the inlet (X0), the far field (Y0, YE, ZE) and the moving
                    floor (Z0), pressure 1 at the outlet (XE), tau=0.51.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import geometry as G

BASE_SEED = 20261203


@dataclass
class BCSpec:
    """One boundary condition, in the user's order. kind: 'noslip',
    'velocity', 'pressure', 'pressure_velocity' on walls; 'map_noslip' on the map."""
    kind: str
    walls: tuple = ()
    p: float = 0.0
    u: tuple = (0.0, 0.0, 0.0)


@dataclass
class Workload:
    name: str
    size: tuple
    q: int
    nu: float
    periodic: tuple = (False, False, False)
    body_force: tuple | None = None
    init_u: tuple = (0.0, 0.0, 0.0)
    bcs: list = field(default_factory=list)
    map: np.ndarray | None = None
    steps: int = 1000
    position: tuple = (0.0, 0.0, 0.0)
    dx: float = 1.0
    info: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return int(np.prod(self.size))


def channel_cylinder(size=(128, 64, 64), radius=8.0, center=(32.0, 32.0), u_in=0.05, nu=0.01, steps=1000,
                     q=19) -> Workload:
    from .lbgk import Block
    block = Block(size, 1.0)
    df = G.normalize(G.generateDFCylinderInf(radius, (0.0, 0.0, 1.0), (center[0], center[1], 0.0)), 1.0)
    m = G.initData(block, df)
    bcs = [BCSpec("velocity", ("X0",), u=(u_in, 0.0, 0.0)),
           BCSpec("pressure", ("XE",), p=1.0),
           BCSpec("noslip", ("Y0", "YE", "Z0", "ZE")),
           BCSpec("map_noslip")]
    return Workload("channel_cylinder_d3q%d_%dx%dx%d" % (q, *size), tuple(size), q, nu, bcs=bcs, map=m,
                    steps=steps, info={"radius": radius, "center": center, "u_in": u_in})


def porous_channel(size=(512, 256, 256), rmin=4.0, rmax=12.0, solid_fraction=0.4, g=1e-6, tau=0.6, steps=5000,
                   seed=BASE_SEED + 2, packer=None) -> Workload:
    """``packer``: a function with the signature of geometry.pack_spheres'
    first six arguments returning (centers, radii), used instead of the
    library's packer (a CPU-only caller that must not load the CUDA library
    passes an equivalent one; the spheres are the same)."""
    from .lbgk import Block
    block = Block(size, 1.0)
    if packer is None:
        pack = G.pack_spheres(size, rmin, rmax, solid_fraction, seed, periodic_x=True)
    else:
        pack = G.SpherePack(*packer(size, rmin, rmax, solid_fraction, seed, True))
    m = G.rasterize_spheres(block, pack, periodic_x=True)
    nu = (tau - 0.5) / 3.0
    solid = float((m[1:-1, 1:-1, 1:-1] <= 0).mean())
    bcs = [BCSpec("noslip", ("Y0", "YE", "Z0", "ZE")), BCSpec("map_noslip")]
    return Workload("porous_channel_d3q19_%dx%dx%d" % tuple(size), tuple(size), 19, nu, periodic=(True, False, False),
                    body_force=(g, 0.0, 0.0), bcs=bcs, map=m, steps=steps,
                    info={"spheres": int(len(pack.radii)), "solid_fraction": solid, "seed": seed, "tau": tau})


def build_lbgk(w: Workload, storage="f32", compVel=True, compRho=True, closure_cls=None, fuse=False,
               packed_rows=False):
    """Instantiate the workload on the GPU through the ASL-style API. With
    ``fuse`` the trailing no-slip conditions (walls and map, which every
    workload lists after its other conditions) are folded into the
    stream-collide kernel."""
    from . import lbgk as A
    vt = {15: A.d3q15(), 19: A.d3q19(), 27: A.d3q27()}[w.q]
    cls = closure_cls or A.LBGK
    block = A.Block(w.size, w.dx, w.position)
    lb = cls(block, w.nu, vt, compVel=compVel, compRho=compRho, storage=storage, periodic=w.periodic,
             body_force=w.body_force, packed_rows=packed_rows)
    lb.init()
    A.LBGKUtilities(lb).initF(w.init_u)
    bcs = []
    for s in w.bcs:
        walls = [getattr(A, n) for n in s.walls]
        if s.kind == "noslip":
            bc = A.generateBCNoSlip(lb, walls)
            if fuse:
                bc.fuse()
            bcs.append(bc)
        elif s.kind == "velocity":
            bcs.append(A.generateBCConstantVelocity(lb, s.u, walls))
        elif s.kind == "pressure":
            bcs.append(A.generateBCConstantPressure(lb, s.p, walls))
        elif s.kind == "pressure_velocity":
            bcs.append(A.generateBCConstantPressureVelocity(lb, s.p, s.u, walls))
        elif s.kind == "map_noslip":
            bc = A.generateBCNoSlip(lb, w.map)
            if fuse:
                bc.fuse()
            bcs.append(bc)
        else:
            raise ValueError(s.kind)
    A.initAll(bcs)
    return lb, bcs


WALL_BITS = {"X0": 1, "XE": 2, "Y0": 4, "YE": 8, "Z0": 16, "ZE": 32}
SLICE_KIND = {"noslip": 0, "velocity": 1, "pressure": 2, "pressure_velocity": 3}


def vehicle_d3q27(size=(768, 384, 384), u_in=0.05, tau=0.51, n_obstacles=12, steps=10000,
                  seed=BASE_SEED + 5) -> Workload:
    """Bluff bodies on a moving floor: boxes (even k) and vertical cylinders
    (odd k) with seeded positions and sizes, all resting on the floor, in the
    upstream half of the tunnel."""
    from .lbgk import Block
    rng = np.random.default_rng(seed)
    nx, ny, nz = size
    block = Block(size, 1.0)
    shapes = []
    for k in range(n_obstacles):
        cx = rng.uniform(0.15, 0.55) * nx
        cy = rng.uniform(0.2, 0.8) * ny
        if k % 2 == 0:
            h = np.array([rng.uniform(0.02, 0.05) * nx, rng.uniform(0.03, 0.08) * ny, rng.uniform(0.06, 0.2) * nz])
            c = np.array([cx, cy, h[2] - 0.5])  # bottom face half a cell below the first interior layer
            shapes.append((G.generateDFBox(c, h), c - h, c + h))
        else:
            r = rng.uniform(0.02, 0.05) * ny
            hgt = rng.uniform(0.1, 0.3) * nz
            c = np.array([cx, cy, hgt / 2 - 0.5])
            shapes.append((G.generateDFCylinder(r, (0.0, 0.0, hgt), c), c - np.array([r, r, hgt / 2]),
                           c + np.array([r, r, hgt / 2])))
    m = G.rasterize_union(block, shapes)
    nu = (tau - 0.5) / 3.0
    u = (u_in, 0.0, 0.0)
    bcs = [BCSpec("velocity", ("X0", "Y0", "YE", "ZE", "Z0"), u=u),
           BCSpec("pressure", ("XE",), p=1.0),
           BCSpec("map_noslip")]
    solid = float((m[1:-1, 1:-1, 1:-1] <= 0).mean())
    return Workload("vehicle_d3q27_%dx%dx%d" % tuple(size), tuple(size), 27, nu, bcs=bcs, map=m, steps=steps,
                    init_u=u, info={"obstacles": n_obstacles, "solid_fraction": solid, "seed": seed, "tau": tau,
                                    "u_in": u_in})


def batch_channels(n=256, steps=2000, seed=BASE_SEED + 3) -> list:
    """The many-small-domains case: n seeded channels of random size, each
    with one box or sphere obstacle (alternating) in its upstream half."""
    from .lbgk import Block
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        size = (int(rng.integers(32, 129)), int(rng.integers(32, 65)), int(rng.integers(32, 65)))
        nx, ny, nz = size
        u_in = float(rng.uniform(0.02, 0.08))
        tau = float(rng.uniform(0.52, 0.8))
        cx, cy, cz = rng.uniform(0.25, 0.45) * nx, rng.uniform(0.35, 0.65) * ny, rng.uniform(0.35, 0.65) * nz
        r = float(rng.uniform(0.12, 0.22)) * min(ny, nz)
        block = Block(size, 1.0)
        if i % 2 == 0:
            c = np.array([cx, cy, cz])
            h = np.array([r, r, r])
            shape = (G.generateDFBox(c, h), c - h, c + h)
        else:
            c = np.array([cx, cy, cz])
            shape = (G.generateDFSphere(r, c), c - r, c + r)
        m = G.rasterize_union(block, [shape])
        u = (u_in, 0.0, 0.0)
        bcs = [BCSpec("velocity", ("X0",), u=u), BCSpec("pressure", ("XE",), p=1.0),
               BCSpec("noslip", ("Y0", "YE", "Z0", "ZE")), BCSpec("map_noslip")]
        out.append(Workload("batch_channel_%d_%dx%dx%d" % (i, *size), size, 19, (tau - 0.5) / 3.0, bcs=bcs, map=m,
                            steps=steps, init_u=u, info={"tau": tau, "u_in": u_in, "obstacle": "box" if i % 2 == 0
                                                         else "sphere"}))
    return out


def build_batch(ws, storage="f32", fuse=True, packed_rows=True):
    """All workloads of a batch on the GPU plus the Batch that steps them
    (short z rows: packed by default)."""
    from . import lbgk as A
    lbs, bcs = [], []
    for w in ws:
        lb, bc = build_lbgk(w, storage=storage, compVel=False, compRho=False, fuse=fuse, packed_rows=packed_rows)
        lbs.append(lb)
        bcs.append(bc)
    return A.Batch(lbs), lbs, bcs
