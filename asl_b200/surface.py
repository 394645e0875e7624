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


# ---- VTK XML PolyData (.vtp) ------------------------------------------------
#
# The .vtp branch of readSurface (aslVTKFormatReaders.cxx:219-257 reads it with
# vtkXMLPolyDataReader). Points and polygons are read from the file's
# DataArrays in any of VTK's encodings: ascii, binary (base64 with a UInt32 or
# UInt64 size header), appended (raw or base64), optionally compressed in
# zlib blocks (vtkZLibDataCompressor); polygons are split into fans of
# triangles.

_VTK_TYPES = {"Float32": "<f4", "Float64": "<f8", "Int8": "<i1", "UInt8": "<u1", "Int16": "<i2", "UInt16": "<u2",
              "Int32": "<i4", "UInt32": "<u4", "Int64": "<i8", "UInt64": "<u8"}


def _vtp_block(raw: bytes, pos: int, hdt: str, compressed: bool, b64: bool):
    """Decode one binary data block starting at raw[pos:]; returns (bytes, next pos)."""
    import base64
    import zlib
    hsz = np.dtype(hdt).itemsize
    if not b64:
        if not compressed:
            n = int(np.frombuffer(raw[pos:pos + hsz], hdt)[0])
            return raw[pos + hsz:pos + hsz + n], pos + hsz + n
        nb = int(np.frombuffer(raw[pos:pos + hsz], hdt)[0])
        head = np.frombuffer(raw[pos:pos + hsz * (3 + nb)], hdt)
        sizes = head[3:3 + nb].astype(np.int64)
        q = pos + hsz * (3 + nb)
        out = b"".join(zlib.decompress(raw[q + int(o):q + int(o) + int(sz)])
                       for o, sz in zip(np.concatenate([[0], np.cumsum(sizes)[:-1]]), sizes))
        return out, q + int(sizes.sum())
    # base64: the text runs to the next tag; arrays of an appended section
    # follow each other, so only the characters this block needs are decoded
    text = b"".join(raw[pos:].split(b"<", 1)[0].split())

    def dec(chars: int) -> bytes:
        return base64.b64decode(text[:chars])
    if not compressed:
        n = int(np.frombuffer(dec(((hsz + 2) // 3) * 4)[:hsz], hdt)[0])
        return dec(((hsz + n + 2) // 3) * 4)[hsz:hsz + n], len(raw)
    # compressed: the header is encoded on its own, then the blocks
    nb = int(np.frombuffer(dec(((hsz + 2) // 3) * 4)[:hsz], hdt)[0])
    hlen = ((hsz * (3 + nb) + 2) // 3) * 4
    head = np.frombuffer(dec(hlen)[:hsz * (3 + nb)], hdt)
    sizes = head[3:3 + nb].astype(np.int64)
    total = int(sizes.sum())
    body = base64.b64decode(text[hlen:hlen + ((total + 2) // 3) * 4])
    out, q = [], 0
    for sz in sizes:
        out.append(zlib.decompress(body[q:q + int(sz)]))
        q += int(sz)
    return b"".join(out), len(raw)


def readVTP(path: str) -> np.ndarray:
    """Triangles of a VTK XML PolyData file, (n, 3, 3) float32 in file coordinates."""
    import re
    with open(path, "rb") as f:
        raw = f.read()
    head_end = raw.find(b"<AppendedData")
    head = raw[: head_end if head_end >= 0 else len(raw)].decode("latin-1")
    root = re.search(r"<VTKFile([^>]*)>", head)
    if not root or 'type="PolyData"' not in root.group(1):
        raise L.ASLError("ASL ERROR: readVTP: not a VTK XML PolyData file")
    attrs = root.group(1)
    hdt = "<u8" if 'header_type="UInt64"' in attrs else "<u4"
    if 'byte_order="BigEndian"' in attrs:
        raise L.ASLError("ASL ERROR: readVTP: big-endian files are not supported")
    compressed = "vtkZLibDataCompressor" in attrs
    app_start, app_b64 = None, False
    if head_end >= 0:
        m = re.match(rb"<AppendedData[^>]*encoding=\"(\w+)\"[^>]*>", raw[head_end:])
        app_b64 = bool(m) and m.group(1) == b"base64"
        app_start = raw.index(b"_", head_end) + 1

    def array(section: str, name: str | None):
        sec = re.search(r"<%s>(.*?)</%s>" % (section, section), head, re.S)
        if not sec:
            raise L.ASLError("ASL ERROR: readVTP: no %s section" % section)
        for m in re.finditer(r"<DataArray([^>]*[^/])>(.*?)</DataArray>|<DataArray([^>]*)/>", sec.group(1), re.S):
            at = m.group(1) or m.group(3)
            if name is not None and ('Name="%s"' % name) not in at:
                continue
            vt = re.search(r'type="(\w+)"', at).group(1)
            fmt = re.search(r'format="(\w+)"', at).group(1)
            dt = _VTK_TYPES[vt]
            if fmt == "ascii":
                return np.array((m.group(2) or "").split(), dtype=dt)
            if fmt == "binary":
                body = (m.group(2) or "").encode()
                data, _ = _vtp_block(body, 0, hdt, compressed, True)
                return np.frombuffer(data, dt)
            if app_start is None:
                raise L.ASLError("ASL ERROR: readVTP: appended array without an AppendedData section")
            off = int(re.search(r'offset="(\d+)"', at).group(1))
            data, _ = _vtp_block(raw, app_start + off, hdt, compressed, app_b64)
            return np.frombuffer(data, dt)
        raise L.ASLError("ASL ERROR: readVTP: array %s of %s not found" % (name, section))

    pts = array("Points", None).astype(np.float32).reshape(-1, 3)
    conn = array("Polys", "connectivity").astype(np.int64)
    offs = array("Polys", "offsets").astype(np.int64)
    tris = []
    start = 0
    for end in offs:
        poly = conn[start:end]
        for k in range(1, len(poly) - 1):
            tris.append((poly[0], poly[k], poly[k + 1]))
        start = end
    if not tris:
        return np.zeros((0, 3, 3), dtype=np.float32)
    return np.ascontiguousarray(pts[np.asarray(tris)], dtype=np.float32)


def writeVTP(path: str, tri: np.ndarray, encoding: str = "appended", compress: bool = False):
    """Write triangles (n, 3, 3) as VTK XML PolyData: encoding "ascii",
    "binary" (base64) or "appended" (raw); zlib-compressed blocks with
    ``compress`` (binary encodings). Points are not merged."""
    import base64
    import struct
    import zlib
    tri = np.asarray(tri, dtype=np.float32).reshape(-1, 3, 3)
    pts = tri.reshape(-1, 3)
    conn = np.arange(len(pts), dtype=np.int64)
    offs = np.arange(3, len(pts) + 1, 3, dtype=np.int64)
    arrays = [("Points", None, "Float32", pts.reshape(-1), 3), ("Polys", "connectivity", "Int64", conn, 1),
              ("Polys", "offsets", "Int64", offs, 1)]

    def block(a: np.ndarray) -> bytes:
        raw = a.tobytes()
        if not compress:
            return struct.pack("<Q", len(raw)) + raw
        z = zlib.compress(raw)
        return struct.pack("<QQQQ", 1, len(raw), len(raw), len(z)) + z

    comp = ' compressor="vtkZLibDataCompressor"' if compress and encoding != "ascii" else ""
    out = ['<?xml version="1.0"?>\n<VTKFile type="PolyData" version="1.0" byte_order="LittleEndian" '
           'header_type="UInt64"%s>\n  <PolyData>\n    <Piece NumberOfPoints="%d" NumberOfPolys="%d">\n'
           % (comp, len(pts), len(tri))]
    appended, off = [], 0
    for section in ("Points", "Polys"):
        out.append("      <%s>\n" % section)
        for sec, name, vt, a, nc in arrays:
            if sec != section:
                continue
            nm = ' Name="%s"' % name if name else ""
            ncs = ' NumberOfComponents="3"' if nc == 3 else ""
            if encoding == "ascii":
                out.append('        <DataArray type="%s"%s%s format="ascii">%s</DataArray>\n'
                           % (vt, nm, ncs, " ".join(repr(float(v)) if vt == "Float32" else str(int(v)) for v in a)))
            elif encoding == "binary":
                b = block(a)
                if compress:  # header and blocks encoded separately, as VTK does
                    hl = 8 * 4
                    txt = base64.b64encode(b[:hl]) + base64.b64encode(b[hl:])
                else:
                    txt = base64.b64encode(b)
                out.append('        <DataArray type="%s"%s%s format="binary">%s</DataArray>\n'
                           % (vt, nm, ncs, txt.decode()))
            else:
                b = block(a)
                out.append('        <DataArray type="%s"%s%s format="appended" offset="%d"/>\n' % (vt, nm, ncs, off))
                appended.append(b)
                off += len(b)
        out.append("      </%s>\n" % section)
    out.append("    </Piece>\n  </PolyData>\n")
    with open(path, "wb") as f:
        f.write("".join(out).encode())
        if appended:
            f.write(b'  <AppendedData encoding="raw">\n   _' + b"".join(appended) + b"\n  </AppendedData>\n")
        f.write(b"</VTKFile>\n")


def readSurface(fileName: str, b: Union[Block, float], *offsets, solid_interior: bool = False) -> SurfaceData:
    """readSurface (aslVTKFormatReaders.cxx:307-345): .stl or .vtp."""
    ext = os.path.splitext(fileName)[1].lower()
    if ext == ".stl":
        tri = readSTL(fileName)
    elif ext == ".vtp":
        tri = readVTP(fileName)
    else:
        raise L.ASLError("ASL ERROR: Reader: file format not supported")
    return surfaceToData(tri, b, *offsets, solid_interior=solid_interior)
