"""CPU tests of the .vti writer (ASL WriterVTKXML layout) and its reader."""
import re
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from asl_b200.lbgk import Block
from asl_b200.writers import WriterVTKXML, read_vti, write_vti


def _header(path):
    buf = open(path, "rb").read()
    head = buf[:buf.index(b"<AppendedData")].decode()
    # close the open elements so the header parses as XML
    return ET.fromstring(head.split("?>", 1)[1] + "</VTKFile>")


def test_roundtrip_ghosted_fields(tmp_path):
    rng = np.random.default_rng(7)
    b = Block((5, 4, 3), dx=0.5, position=(1.0, 2.0, 3.0))
    rho = rng.standard_normal(b.ghosted)
    u = rng.standard_normal((3, *b.ghosted))
    w = WriterVTKXML(str(tmp_path / "flow"), b)
    w.addScalars("rho", rho)
    w.addVector("u", lambda: u)
    p0 = w.write()
    p1 = w.write()
    assert p0.endswith("flow_0.vti") and p1.endswith("flow_1.vti") and w.numOfWrites == 2
    d = read_vti(p0)
    assert d["rho"].dtype == np.float64  # FP64 fields stay FP64
    assert np.array_equal(d["rho"], rho[1:-1, 1:-1, 1:-1])
    assert np.array_equal(d["u"], u[:, 1:-1, 1:-1, 1:-1])


def test_axes_and_components_reversed(tmp_path):
    b = Block((4, 3, 2), dx=2.0, position=(10.0, 20.0, 30.0))
    x, y, z = np.meshgrid(np.arange(4), np.arange(3), np.arange(2), indexing="ij")
    u = np.stack([x, y, z]).astype(np.float32)
    w = WriterVTKXML(str(tmp_path / "ax"), b)
    w.addScalars("x", x.astype(np.float32))
    w.addVector("u", u)
    path = w.write()
    root = _header(path)
    img = root.find("ImageData")
    # VTK x is ASL z: extents and origin come reversed
    assert img.get("WholeExtent") == "0 1 0 2 0 3"
    assert [float(v) for v in img.get("Origin").split()] == [30.0, 20.0, 10.0]
    assert [float(v) for v in img.get("Spacing").split()] == [2.0, 2.0, 2.0]
    assert root.get("type") == "ImageData" and root.get("header_type") == "UInt64"
    pd = img.find("Piece/PointData")
    assert pd.get("Scalars") == "x"
    arrays = pd.findall("DataArray")
    assert [a.get("Name") for a in arrays] == ["x", "u"]
    assert arrays[1].get("NumberOfComponents") == "3"
    # raw layout: first point is ASL (0,0,0); the second point is VTK x + 1 = ASL z + 1,
    # and each point's first component is ASL's component 2 (z)
    buf = open(path, "rb").read()
    data0 = buf.index(b"_", buf.index(b"<AppendedData")) + 1
    off = int(arrays[1].get("offset"))
    raw = np.frombuffer(buf[data0 + off + 8:data0 + off + 8 + 24 * 4 * 3], dtype=np.float32).reshape(-1, 3)
    assert raw[1].tolist() == [1.0, 0.0, 0.0]   # point (x 0, y 0, z 1): components (z, y, x)
    assert raw[2].tolist() == [0.0, 1.0, 0.0]   # point (x 0, y 1, z 0)
    assert raw[6].tolist() == [0.0, 0.0, 1.0]   # point (x 1, y 0, z 0)
    d = read_vti(path)
    assert np.array_equal(d["u"], u) and np.array_equal(d["x"], x)


def test_errors(tmp_path):
    b = Block((4, 4, 4))
    w = WriterVTKXML(str(tmp_path / "e"), b)
    with pytest.raises(ValueError, match="no fields"):
        w.write()
    w.addScalars("bad", np.zeros((5, 5, 5)))
    with pytest.raises(ValueError, match="shape"):
        w.write()
    w2 = WriterVTKXML(str(tmp_path / "e2"), b)
    w2.addVector("v", np.zeros((4, 4, 4)))
    with pytest.raises(ValueError, match="3 components"):
        w2.write()


def test_write_vti_without_block(tmp_path):
    a = np.arange(24, dtype=np.float32).reshape(2, 3, 4)
    path = str(tmp_path / "plain.vti")
    write_vti(path, a.shape, (0, 0, 0), 1.0, [("a", 1, a)])
    text = open(path, "rb").read()
    assert re.search(rb'WholeExtent="0 3 0 2 0 1"', text)
    assert np.array_equal(read_vti(path)["a"], a)
