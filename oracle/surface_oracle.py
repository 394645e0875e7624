"""CPU oracle for surface distance maps (test infrastructure only).

Checks the CUDA sampling behind readSurface. ASL samples the distance with
VTK's vtkImplicitModeller (src/readers/aslVTKFormatReaders.cxx:136-210); VTK is
a third-party dependency that is neither vendored in the reference nor
installed here (no pinned version), so this oracle restates the quantity VTK
computes per voxel in that mode — the distance from the sample point to the
closest point of the nearest triangle — by brute force in FP64, and the
inside test of the solid-interior extension by ray parity. Parity against
VTK itself is unpinned; the oracle is pinned by known answers in the tests
(distances to a box and to a polyhedral sphere, inside/outside of closed
meshes).
"""
from __future__ import annotations

import numpy as np


def point_triangle_distance(p: np.ndarray, tri: np.ndarray) -> np.ndarray:
    """Distance of points p (m, 3) to one triangle (3, 3): projection onto
    the plane when it falls inside, else the nearest of the three edges
    (segments, clamped)."""
    p = np.asarray(p, dtype=np.float64)
    a, b, c = (np.asarray(v, dtype=np.float64) for v in tri)
    n = np.cross(b - a, c - a)
    nn = n @ n
    best = np.full(len(p), np.inf)
    if nn > 0:
        t = ((p - a) @ n) / nn
        q = p - t[:, None] * n
        inside = np.ones(len(p), dtype=bool)
        for u, v in ((a, b), (b, c), (c, a)):
            inside &= (np.cross(v - u, q - u) @ n) >= 0
        d = np.abs(t) * np.sqrt(nn)
        best = np.where(inside, d, best)
    for u, v in ((a, b), (b, c), (c, a)):
        e = v - u
        ee = e @ e
        s = np.clip(((p - u) @ e) / ee, 0.0, 1.0) if ee > 0 else np.zeros(len(p))
        d = np.linalg.norm(p - (u + s[:, None] * e), axis=1)
        best = np.minimum(best, d)
    return best


def distance_field(tris: np.ndarray, size, pos0, dx: float) -> np.ndarray:
    """Unsigned distance at every cell (i, j, k) -> pos0 + (i, j, k) dx."""
    gx, gy, gz = size
    ax = [pos0[a] + np.arange((gx, gy, gz)[a], dtype=np.float64) * dx for a in range(3)]
    pts = np.stack(np.meshgrid(*ax, indexing="ij"), axis=-1).reshape(-1, 3)
    d = np.full(len(pts), np.inf)
    for t in np.asarray(tris, dtype=np.float64).reshape(-1, 3, 3):
        d = np.minimum(d, point_triangle_distance(pts, t))
    return d.reshape(gx, gy, gz)


def inside_parity(tris: np.ndarray, size, pos0, dx: float) -> np.ndarray:
    """True where a ray from the cell towards -x crosses the surface an odd
    number of times (points exactly on an edge are not generated by the tests)."""
    gx, gy, gz = size
    ys = pos0[1] + np.arange(gy) * dx
    zs = pos0[2] + np.arange(gz) * dx
    xs = pos0[0] + np.arange(gx) * dx
    Y, Z = np.meshgrid(ys, zs, indexing="ij")
    count = np.zeros((gx, gy, gz), dtype=np.int64)
    for t in np.asarray(tris, dtype=np.float64).reshape(-1, 3, 3):
        a, b, c = t
        area = (b[1] - a[1]) * (c[2] - a[2]) - (b[2] - a[2]) * (c[1] - a[1])
        if area == 0:
            continue
        w0 = (b[1] - a[1]) * (Z - a[2]) - (b[2] - a[2]) * (Y - a[1])
        w1 = (c[1] - b[1]) * (Z - b[2]) - (c[2] - b[2]) * (Y - b[1])
        w2 = (a[1] - c[1]) * (Z - c[2]) - (a[2] - c[2]) * (Y - c[1])
        s = np.sign(area)
        hit = (w0 * s > 0) & (w1 * s > 0) & (w2 * s > 0)
        xc = a[0] + (w2 * (b[0] - a[0]) + w0 * (c[0] - a[0])) / area
        count += (hit[None] & (xs[:, None, None] > xc[None])).astype(np.int64)
    return (count % 2) == 1


def box_mesh(lo, hi) -> np.ndarray:
    """12 outward-oriented triangles of the axis-aligned box [lo, hi]."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    v = np.array([[lo[0] if i & 1 == 0 else hi[0], lo[1] if i & 2 == 0 else hi[1], lo[2] if i & 4 == 0 else hi[2]]
                  for i in range(8)])
    quads = [(0, 2, 6, 4), (1, 5, 7, 3), (0, 4, 5, 1), (2, 3, 7, 6), (0, 1, 3, 2), (4, 6, 7, 5)]
    tris = []
    for q in quads:
        tris.append([v[q[0]], v[q[1]], v[q[2]]])
        tris.append([v[q[0]], v[q[2]], v[q[3]]])
    return np.asarray(tris, dtype=np.float32)


def icosphere(radius: float, center, subdiv: int = 2) -> np.ndarray:
    """Triangulated sphere: an icosahedron subdivided ``subdiv`` times, the
    vertices pushed onto the sphere."""
    t = (1 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.asarray(p, float) / np.linalg.norm(p) for p in v]
    for _ in range(subdiv):
        cache = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]
        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    V = np.asarray(verts) * radius + np.asarray(center, float)
    return V[np.asarray(f)].astype(np.float32)
