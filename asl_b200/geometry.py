"""Signed distance functions and their rasterisation onto a ghosted block.

Follows ASL's DistanceFunction family (src/math/aslDistanceFunction.cxx and
src/aslGeomInc.cxx of AvtechScientific/ASL): distances are negative inside a
solid, union is min (``|``), intersection is max (``&``), inversion is ``-``,
and ``normalize(df, dx)`` clips df / (1.8 dx) to [-1, 1]. ``initData``
evaluates a function at the physical position of every ghosted cell, in FP32
like ASL's generated kernels (src/aslGeomInc.cxx:197-219).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

NORMALIZATION_SCALE = 1.8  # DistFNormalization::scaleFactor (aslDistanceFunction.cxx:142)


class DistanceFunction:
    def distance(self, pos: np.ndarray) -> np.ndarray:  # pos: (3, ...) float32
        raise NotImplementedError

    # An operand that is None leaves the other one, as ASL's operators do
    # with an uninitialised SPDistanceFunction (aslGeomInc.cxx:39-66), so a
    # union can be built up from nothing.
    def __or__(self, other):  # union
        return self if other is None else _Binary(self, other, np.minimum)

    def __ror__(self, other):
        return self if other is None else _Binary(other, self, np.minimum)

    def __and__(self, other):  # intersection
        return self if other is None else _Binary(self, other, np.maximum)

    def __rand__(self, other):
        return self if other is None else _Binary(other, self, np.maximum)

    def __neg__(self):
        return _Unary(self, lambda d: -d)


class _Binary(DistanceFunction):
    def __init__(self, a, b, op):
        self.a, self.b, self.op = a, b, op

    def distance(self, pos):
        return self.op(self.a.distance(pos), self.b.distance(pos))


class _Unary(DistanceFunction):
    def __init__(self, a, fn):
        self.a, self.fn = a, fn

    def distance(self, pos):
        return self.fn(self.a.distance(pos))


def _f32(v):
    return np.asarray(v, dtype=np.float32).reshape(3, *([1] * 0))


class DFSphere(DistanceFunction):
    """|p - c| - r (aslDistanceFunction.cxx:92-104)."""

    def __init__(self, r, c):
        self.r = np.float32(r)
        self.c = np.asarray(c, dtype=np.float32)

    def distance(self, pos):
        d = pos - self.c.reshape(3, *([1] * (pos.ndim - 1)))
        return np.sqrt((d * d).sum(0)) - self.r


class DFCylinderInf(DistanceFunction):
    """Infinite cylinder: |(p-c) - ((p-c).l) l| - r (aslDistanceFunction.cxx:104-114)."""

    def __init__(self, r, l, c):
        l = np.asarray(l, dtype=np.float64)
        self.r = np.float32(r)
        self.l = (l / np.linalg.norm(l)).astype(np.float32)
        self.c = np.asarray(c, dtype=np.float32)

    def distance(self, pos):
        sh = (3, *([1] * (pos.ndim - 1)))
        d = pos - self.c.reshape(sh)
        proj = (d * self.l.reshape(sh)).sum(0)
        v = d - proj[None] * self.l.reshape(sh)
        return np.sqrt((v * v).sum(0)) - self.r


class DFPlane(DistanceFunction):
    """p.n/|n| - p0.n/|n| (aslDistanceFunction.cxx:130-140)."""

    def __init__(self, n, p0):
        n = np.asarray(n, dtype=np.float64)
        nn = n / math.sqrt(float((n * n).sum()))
        self.n = nn.astype(np.float32)
        self.b = np.float32(np.dot(np.asarray(p0, dtype=np.float64), n) / math.sqrt(float((n * n).sum())))

    def distance(self, pos):
        sh = (3, *([1] * (pos.ndim - 1)))
        return (pos * self.n.reshape(sh)).sum(0) - self.b


class _Normalized(DistanceFunction):
    def __init__(self, a, dx):
        self.a = a
        self.factor = np.float32(1.0 / dx / NORMALIZATION_SCALE)

    def distance(self, pos):
        d = self.factor * self.a.distance(pos)
        d = np.where(d > 1.0, np.float32(1.0), d)
        return np.where(d < -1.0, np.float32(-1.0), d).astype(np.float32)


def generateDFSphere(r, c) -> DistanceFunction:
    return DFSphere(r, c)


def generateDFCylinderInf(r, l, c) -> DistanceFunction:
    return DFCylinderInf(r, l, c)


def generateDFPlane(n, p0) -> DistanceFunction:
    return DFPlane(n, p0)


def generateDFCylinder(r, l, c) -> DistanceFunction:
    """Finite cylinder of axis vector l (its length is the height), aslGeomInc.cxx:98-106."""
    l = np.asarray(l, dtype=np.float64)
    c = np.asarray(c, dtype=np.float64)
    return DFCylinderInf(r, l, c) & DFPlane(l, c + l * 0.5) & DFPlane(-l, c - l * 0.5)


def generateDFBox(center, half) -> DistanceFunction:
    """Axis-aligned box as the intersection of six planes (an extension built the
    way generateDFConvexPolygonPrism builds prisms, aslGeomInc.cxx:123-140)."""
    c = np.asarray(center, dtype=np.float64)
    h = np.asarray(half, dtype=np.float64)
    res = None
    for a in range(3):
        e = np.zeros(3)
        e[a] = 1.0
        pair = DFPlane(e, c + h * e) & DFPlane(-e, c - h * e)
        res = pair if res is None else (res & pair)
    return res


def normalize(df: DistanceFunction, dx: float) -> DistanceFunction:
    return _Normalized(df, dx)


def block_positions(block) -> np.ndarray:
    """Positions of the ghosted cells in FP32, shape (3, gx, gy, gz)."""
    gx, gy, gz = block.ghosted
    axes = [np.float32(block.position[a]) + (np.arange((gx, gy, gz)[a], dtype=np.float32) - np.float32(1.0))
            * np.float32(block.dx) for a in range(3)]
    return np.stack(np.meshgrid(*axes, indexing="ij")).astype(np.float32)


def initData(block, df: DistanceFunction) -> np.ndarray:
    """Rasterise a distance function onto the ghosted block (float32 map)."""
    return np.ascontiguousarray(df.distance(block_positions(block)).astype(np.float32))


# ---- seeded porous medium (random non-overlapping spheres) -------------------

@dataclass
class SpherePack:
    centers: np.ndarray  # (n, 3), interior-cell coordinates (cell i at position i)
    radii: np.ndarray    # (n,)


def pack_spheres(size, rmin: float, rmax: float, solid_fraction: float, seed: int, periodic_x: bool = True,
                 attempts: int = 400) -> SpherePack:
    """Random sequential addition of non-overlapping spheres, radii U[rmin, rmax],
    placed largest first until the sphere volume reaches ``solid_fraction`` of
    the box. Spheres stay inside y/z; x is periodic when ``periodic_x``.
    Runs in the library's host code (aslb_geom_pack_spheres)."""
    import ctypes as C
    from . import _lib as L
    nx, ny, nz = size
    cap = int(solid_fraction * nx * ny * nz / (4.0 / 3.0 * math.pi * rmin ** 3)) + 16
    centers = np.zeros((cap, 3))
    radii = np.zeros(cap)
    n = C.c_int(0)
    L.check(L.load().aslb_geom_pack_spheres(int(nx), int(ny), int(nz), float(rmin), float(rmax), float(solid_fraction),
                                            int(seed), int(bool(periodic_x)), int(attempts), cap,
                                            centers.ctypes.data_as(L._pd), radii.ctypes.data_as(L._pd), C.byref(n)),
            "pack_spheres")
    return SpherePack(centers[:n.value].copy(), radii[:n.value].copy())


def rasterize_spheres(block, pack: SpherePack, periodic_x: bool = True, margin: float = 2.0) -> np.ndarray:
    """normalize(union of spheres, dx) on the ghosted block without evaluating
    every sphere everywhere: each sphere updates its bounding box only (cells
    farther than 1.8 dx from every surface clip to +1 anyway)."""
    gx, gy, gz = block.ghosted
    nx = block.size[0]
    m = np.ones((gx, gy, gz), dtype=np.float32)
    scale = np.float32(1.0 / (block.dx * NORMALIZATION_SCALE))
    for c, r in zip(pack.centers, pack.radii):
        ext = r + margin
        lo = [int(math.floor(c[a] - ext)) + 1 for a in range(3)]
        hi = [int(math.ceil(c[a] + ext)) + 1 for a in range(3)]
        shifts = [0]
        if periodic_x:
            shifts = [-nx, 0, nx]
        for sx in shifts:
            x0, x1 = max(lo[0] + sx, 0), min(hi[0] + sx, gx - 1)
            y0, y1 = max(lo[1], 0), min(hi[1], gy - 1)
            z0, z1 = max(lo[2], 0), min(hi[2], gz - 1)
            if x0 > x1 or y0 > y1 or z0 > z1:
                continue
            xs = (np.arange(x0, x1 + 1, dtype=np.float32) - 1 - np.float32(sx) - np.float32(c[0]))
            ys = (np.arange(y0, y1 + 1, dtype=np.float32) - 1 - np.float32(c[1]))
            zs = (np.arange(z0, z1 + 1, dtype=np.float32) - 1 - np.float32(c[2]))
            d = np.sqrt(xs[:, None, None] ** 2 + ys[None, :, None] ** 2 + zs[None, None, :] ** 2) - np.float32(r)
            d = np.clip(d * scale, -1.0, 1.0).astype(np.float32)
            sub = m[x0:x1 + 1, y0:y1 + 1, z0:z1 + 1]
            np.minimum(sub, d, out=sub)
    return m


def rasterize_union(block, shapes, margin: float = 2.0) -> np.ndarray:
    """normalize(union of shapes, dx) on the ghosted block, evaluating each
    shape only inside its bounding box grown by ``margin`` cells (outside it the
    normalised distance is clipped to +1 anyway). ``shapes``: (df, lo, hi) with
    lo / hi the physical corners of the shape's bounding box."""
    gx, gy, gz = block.ghosted
    m = np.ones((gx, gy, gz), dtype=np.float32)
    dx = float(block.dx)
    for df, lo, hi in shapes:
        nd = normalize(df, dx)
        idx_lo = [max(int(math.floor((lo[a] - block.position[a]) / dx - margin)) + 1, 0) for a in range(3)]
        idx_hi = [min(int(math.ceil((hi[a] - block.position[a]) / dx + margin)) + 1, (gx, gy, gz)[a] - 1)
                  for a in range(3)]
        if any(idx_lo[a] > idx_hi[a] for a in range(3)):
            continue
        axes = [np.float32(block.position[a]) + (np.arange(idx_lo[a], idx_hi[a] + 1, dtype=np.float32)
                                                 - np.float32(1.0)) * np.float32(dx) for a in range(3)]
        pos = np.stack(np.meshgrid(*axes, indexing="ij")).astype(np.float32)
        sub = m[idx_lo[0]:idx_hi[0] + 1, idx_lo[1]:idx_hi[1] + 1, idx_lo[2]:idx_hi[2] + 1]
        np.minimum(sub, nd.distance(pos), out=sub)
    return m
