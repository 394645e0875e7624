"""Output and restart files without VTK.

``WriterVTKXML`` mirrors ASL's writer (src/writers/aslWriter.h:44-72,
src/writers/aslVTKFormatWriters.cxx:43-126): ``addScalars`` / ``addVector``
register fields, every ``write()`` produces ``<file>_<n>.vti``, a VTK XML
ImageData file with appended raw binary data. Like ASL's casts
(src/utilities/aslVTKCasters.cxx:166-181) the axes are reversed — ASL's
arrays are z fastest, VTK's x fastest, so VTK's x is ASL's z — and so are
the vector components (ASL writes component 2 first). The interior cells are
written (ghost layers dropped); values are FP32 (FP64 fields stay FP64).

``save_checkpoint`` / ``load_checkpoint`` dump and restore a domain's
population array as stored, with its step count and AA parity, the role of
ASL's ABD restart dumps (src/writers/aslABDFormat.h:45-137).
"""
from __future__ import annotations

import os
import struct
from typing import Callable, Union

import numpy as np

Source = Union[np.ndarray, Callable[[], np.ndarray]]


class WriterVTKXML:
    """``WriterVTKXML(file, block)``; fields are arrays in ASL's ghosted or
    interior layout (x, y, z), or callables returning them at write time."""

    def __init__(self, file: str, block=None):
        self.file = file
        self.block = block
        self.scalars: list[tuple[str, Source]] = []
        self.vectors: list[tuple[str, Source]] = []
        self.numOfWrites = 0

    def addScalars(self, name: str, data: Source):
        self.scalars.append((name, data))

    def addVector(self, name: str, data: Source):
        self.vectors.append((name, data))

    def _interior(self, a: np.ndarray, ncomp: int) -> np.ndarray:
        a = np.asarray(a)
        if ncomp == 3 and a.ndim == 3:
            raise ValueError("WriterVTKXML: a vector field needs 3 components")
        shape = a.shape[-3:]
        if self.block is not None:
            size = tuple(self.block.size)
            if shape == tuple(s + 2 for s in size):
                a = a[..., 1:-1, 1:-1, 1:-1]
            elif shape != size:
                raise ValueError("WriterVTKXML: field of shape %s on a block of %s" % (shape, size))
        return a

    def write(self) -> str:
        if not self.scalars and not self.vectors:
            raise ValueError("WriterVTKXML::write() - there are no fields to write")
        arrays = []
        for name, src in self.scalars:
            a = self._interior(src() if callable(src) else src, 1)
            arrays.append((name, 1, a))
        for name, src in self.vectors:
            a = self._interior(src() if callable(src) else src, 3)
            arrays.append((name, 3, a))
        nx, ny, nz = arrays[0][2].shape[-3:]
        pos = tuple(self.block.position) if self.block is not None else (0.0, 0.0, 0.0)
        dx = float(self.block.dx) if self.block is not None else 1.0
        path = "%s_%d.vti" % (self.file, self.numOfWrites)
        write_vti(path, (nx, ny, nz), pos, dx, arrays)
        self.numOfWrites += 1
        return path


def write_vti(path: str, size, position, dx: float, arrays):
    """arrays: (name, ncomp, array (ncomp?, nx, ny, nz) in ASL order)."""
    nx, ny, nz = size
    blobs, heads, off = [], [], 0
    for name, ncomp, a in arrays:
        dt = np.float64 if a.dtype == np.float64 else np.float32
        if ncomp == 1:
            data = np.ascontiguousarray(a, dtype=dt).reshape(-1)
        else:
            # point-major, components reversed (VTK x = ASL z)
            data = np.ascontiguousarray(np.stack([a[2], a[1], a[0]], axis=-1), dtype=dt).reshape(-1)
        raw = data.tobytes()
        blobs.append(struct.pack("<Q", len(raw)) + raw)
        vt = "Float64" if dt == np.float64 else "Float32"
        nc = "" if ncomp == 1 else ' NumberOfComponents="3"'
        heads.append('        <DataArray type="%s" Name="%s"%s format="appended" offset="%d"/>\n' % (vt, name, nc, off))
        off += len(blobs[-1])
    ext = "0 %d 0 %d 0 %d" % (nz - 1, ny - 1, nx - 1)
    first = next((n for n, c, _ in arrays if c == 1), None)
    sc = ' Scalars="%s"' % first if first else ""
    head = ('<?xml version="1.0"?>\n'
            '<VTKFile type="ImageData" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n'
            '  <ImageData WholeExtent="%s" Origin="%r %r %r" Spacing="%r %r %r">\n'
            '    <Piece Extent="%s">\n'
            '      <PointData%s>\n%s      </PointData>\n'
            '      <CellData>\n      </CellData>\n'
            '    </Piece>\n'
            '  </ImageData>\n'
            '  <AppendedData encoding="raw">\n   _') % (
        ext, float(position[2]), float(position[1]), float(position[0]), dx, dx, dx, ext, sc, "".join(heads))
    with open(path, "wb") as f:
        f.write(head.encode())
        for b in blobs:
            f.write(b)
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")


def read_vti(path: str) -> dict:
    """Fields of a .vti written by write_vti, back in ASL order (x, y, z)."""
    import re
    with open(path, "rb") as f:
        buf = f.read()
    start = buf.index(b"<AppendedData encoding=\"raw\">")
    head = buf[:start].decode()
    data0 = buf.index(b"_", start) + 1
    ext = [int(v) for v in re.search(r'WholeExtent="([^"]+)"', head).group(1).split()]
    nzv, nyv, nxv = ext[1] + 1, ext[3] + 1, ext[5] + 1
    out = {}
    for m in re.finditer(r'<DataArray type="(\w+)" Name="([^"]+)"( NumberOfComponents="3")? format="appended" '
                         r'offset="(\d+)"/>', head):
        vt, name, vec, off = m.group(1), m.group(2), m.group(3), int(m.group(4))
        p = data0 + off
        n = struct.unpack("<Q", buf[p:p + 8])[0]
        a = np.frombuffer(buf[p + 8:p + 8 + n], dtype=np.float64 if vt == "Float64" else np.float32)
        if vec:
            a = a.reshape(nxv, nyv, nzv, 3)
            out[name] = np.stack([a[..., 2], a[..., 1], a[..., 0]])
        else:
            out[name] = a.reshape(nxv, nyv, nzv)
    return out


def save_checkpoint(lb, path: str) -> str:
    """The domain's population array as stored (its AA representation and
    storage format) with step count and parity: restoring it into a domain
    built the same way (size, lattice, storage, conditions) continues bit
    for bit."""
    data, meta = lb.saveState()
    path = path if path.endswith(".npz") else path + ".npz"
    np.savez(path, state=data, meta=meta, q=np.int64(lb.vectorTemplate.q), size=np.asarray(lb.block.size))
    return path


def load_checkpoint(lb, path: str) -> int:
    """Restore a checkpoint; returns its step count."""
    d = np.load(path if os.path.exists(path) else path + ".npz")
    if int(d["q"]) != lb.vectorTemplate.q or tuple(d["size"]) != tuple(lb.block.size):
        raise ValueError("load_checkpoint: the checkpoint is of another domain")
    lb.loadState(d["state"], d["meta"])
    return int(d["meta"][0])
