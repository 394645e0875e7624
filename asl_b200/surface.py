"""Surfaces to distance maps: ASL's ``readSurface`` without VTK.

ASL (src/readers/aslVTKFormatReaders.h:66-79, .cxx:136-345) reads an STL or
VTP surface, samples the unsigned distance to it on a grid with VTK's
implicit modeller and returns the map (d - offset) / (1.8 dx), whose negative
cells are a solid shell around the surface. Here the STL file is read by the
library (``aslb_read_stl``) and the distance is sampled by its CUDA kernels
(``aslb_surface_map``, exact within a band around the surface). As in ASL the
surface's file coordinates (X, Y, Z) are VTK's axes, whose x is ASL's z: the
surface sits at ASL position (Z, Y, X).

Overloads, as in ASL:
  readSurface(file, block)  samples block.size points from block.position
                            (offset 1.2 dx); the map's internal block is
                            block shrunk by one cell on every side;
  readSurface(file, dx)     samples the surface's bounding box, grown by
                            3.6 dx (offset 1.8 dx);
  readSurface(file, dx, X0, XE, Y0, YE, Z0, ZE)
                            the bounding box grown on each side by that
                            fraction of its extent (offset 1.8 dx).
VTK spreads the samples evenly over the bounds (spacing extent / (n - 1));
here the spacing is dx exactly and the grid starts at the low bound.
``solid_interior`` (an extension) also makes the inside of a closed surface
solid (ray parity along x).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import struct
from typing import Sequence, Union

import numpy as np

from . import _lib as L
from .lbgk import Block

BAND_CELLS = 4.0  # exact distances within this many cells of the surface


class SurfaceData(np.ndarray):
    """A distance map (ghosted FP32 array) that knows its grid, like ASL's
    data container: ``getInternalBlock()`` is the block to simulate on."""

    def __array_finalize__(self, obj):
        self.internal_block = getattr(obj, "internal_block", None)

    def getInternalBlock(self) -> Block:
        return self.internal_block


def readSTL(path: str) -> np.ndarray:
    """Triangles of a binary or ASCII STL file, (n, 3, 3) float32 in file coordinates."""
    lib = L.load()
    n = C.c_longlong()
    L.check(lib.aslb_read_stl(os.fsencode(path), None, 0, C.byref(n)), "readSTL")
    tri = np.empty((n.value, 3, 3), dtype=np.float32)
    L.check(lib.aslb_read_stl(os.fsencode(path), tri.ctypes.data_as(C.c_void_p), n.value, C.byref(n)), "readSTL")
    return tri


def writeSTL(path: str, tri: np.ndarray, binary: bool = True, name: str = "surface"):
    """Write triangles (n, 3, 3) as STL (normals from the vertex order)."""
    tri = np.asarray(tri, dtype=np.float32).reshape(-1, 3, 3)
    nrm = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    ln = np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm = np.where(ln > 0, nrm / np.where(ln > 0, ln, 1), 0).astype(np.float32)
    if binary:
        rec = np.zeros(len(tri), dtype=[("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")])
        rec["n"] = nrm
        rec["v"] = tri.reshape(-1, 9)
        with open(path, "wb") as f:
            f.write(name.encode()[:80].ljust(80, b" "))
            f.write(struct.pack("<I", len(tri)))
            f.write(rec.tobytes())
    else:
        with open(path, "w") as f:
            f.write("solid %s\n" % name)
            for t, n in zip(tri, nrm):
                f.write("  facet normal %r %r %r\n    outer loop\n" % tuple(float(v) for v in n))
                for v in t:
                    f.write("      vertex %r %r %r\n" % tuple(float(c) for c in v))
                f.write("    endloop\n  endfacet\n")
            f.write("endsolid %s\n" % name)


def surface_map(tri_asl: np.ndarray, size: Sequence[int], pos0: Sequence[float], dx: float, offset: float,
                scale: float, solid_interior: bool = False, band: float | None = None) -> np.ndarray:
    """(d - offset) / scale on the size[0] x size[1] x size[2] grid whose cell
    (i, j, k) is at pos0 + (i, j, k) dx; triangles in ASL coordinates."""
    lib = L.load()
    tri = np.ascontiguousarray(tri_asl, dtype=np.float32).reshape(-1, 9)
    gx, gy, gz = (int(s) for s in size)
    out = np.empty((gx, gy, gz), dtype=np.float32)
    band = BAND_CELLS * dx if band is None else float(band)
    L.check(lib.aslb_surface_map(tri.ctypes.data_as(C.c_void_p), len(tri), gx, gy, gz, L.dvec(pos0), float(dx),
                                 band, int(bool(solid_interior)), float(offset), float(scale),
                                 out.ctypes.data_as(C.c_void_p)), "readSurface")
    return out


def _to_asl(tri: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(tri, dtype=np.float32)[..., ::-1])


def _wrap(m: np.ndarray, pos0, dx) -> SurfaceData:
    d = m.view(SurfaceData)
    size = tuple(s - 2 for s in m.shape)
    if min(size) < 1:
        raise L.ASLError("ASL ERROR: readSurface: the sampled grid has no interior")
    d.internal_block = Block(size, dx, tuple(float(p) + dx for p in pos0))
    return d


def surfaceToData(tri, b: Union[Block, float], *offsets, solid_interior: bool = False) -> SurfaceData:
    """The three surfaceToData overloads of aslVTKFormatReaders.cxx:136-210
    on triangles in file coordinates."""
    tri = _to_asl(tri)
    if isinstance(b, Block):
        if offsets:
            raise L.ASLError("ASL ERROR: readSurface: offsets go with the spacing overload")
        dx = b.dx
        m = surface_map(tri, b.size, b.position, dx, 1.2 * dx, 1.8 * dx, solid_interior)
        return _wrap(m, b.position, dx)
    dx = float(b)
    if len(tri) == 0:
        raise L.ASLError("ASL ERROR: readSurface: empty surface")
    flat = tri.reshape(-1, 3).astype(np.float64)
    lo, hi = flat.min(0), flat.max(0)
    if offsets:
        if len(offsets) != 6:
            raise L.ASLError("ASL ERROR: readSurface: six offsets X0, XE, Y0, YE, Z0, ZE")
        ext = hi - lo
        lo = lo - ext * np.asarray(offsets[0::2], dtype=np.float64)
        hi = hi + ext * np.asarray(offsets[1::2], dtype=np.float64)
    else:
        lo, hi = lo - 3.6 * dx, hi + 3.6 * dx
    size = [int(math.floor((hi[a] - lo[a]) / dx)) + 1 for a in range(3)]
    m = surface_map(tri, size, lo, dx, 1.8 * dx, 1.8 * dx, solid_interior)
    return _wrap(m, tuple(lo), dx)


def readSurface(fileName: str, b: Union[Block, float], *offsets, solid_interior: bool = False) -> SurfaceData:
    ext = os.path.splitext(fileName)[1].lower()
    if ext != ".stl":
        raise L.ASLError("ASL ERROR: Reader: file format not supported")
    return surfaceToData(readSTL(fileName), b, *offsets, solid_interior=solid_interior)
