"""CPU tests of the surface oracle (known answers), the STL reader of the
library (host code, no GPU call) and readSurface's argument handling."""
import numpy as np
import pytest

from asl_b200 import surface as S
from oracle import surface_oracle as SO


def test_oracle_box_known_answers():
    box = SO.box_mesh((0, 0, 0), (1, 1, 1))
    pts = np.array([[2.0, 0.5, 0.5], [2.0, 2.0, 0.5], [2.0, 2.0, 2.0], [0.5, 0.5, 0.25], [0.5, 0.5, 0.5]])
    d = np.min([SO.point_triangle_distance(pts, t) for t in box], axis=0)
    assert np.allclose(d, [1.0, 2 ** 0.5, 3 ** 0.5, 0.25, 0.5], atol=1e-12)
    inside = SO.inside_parity(box, (5, 5, 5), (-0.45, -0.43, -0.41), 0.4)
    # cells at -0.45 + 0.4 i (and so on): inside for i = 2 and 3 on every axis
    # (offsets keep the columns off the faces' diagonals)
    want = np.zeros((5, 5, 5), dtype=bool)
    want[2:4, 2:4, 2:4] = True
    assert np.array_equal(inside, want)


def test_oracle_icosphere():
    sph = SO.icosphere(1.0, (0, 0, 0), subdiv=2)
    assert sph.shape == (320, 3, 3)
    assert np.allclose(np.linalg.norm(sph.reshape(-1, 3), axis=1), 1.0, atol=1e-6)
    d = SO.distance_field(sph, (1, 1, 1), (3.0, 0.0, 0.0), 1.0)
    assert 2.0 <= d[0, 0, 0] <= 2.0 + 0.02  # chordal error of the faces
    inside = SO.inside_parity(sph, (3, 1, 1), (-0.31, 0.013, 0.017), 0.7)  # x = -0.31, 0.39, 1.09
    assert inside.ravel().tolist() == [True, True, False]


@pytest.mark.parametrize("binary", [True, False])
def test_stl_roundtrip(tmp_path, binary):
    sph = SO.icosphere(2.0, (1.0, -3.0, 0.5), subdiv=1)
    path = str(tmp_path / ("s_bin.stl" if binary else "s_ascii.stl"))
    S.writeSTL(path, sph, binary=binary)
    got = S.readSTL(path)
    assert got.shape == sph.shape and np.array_equal(got, sph)


def test_stl_errors(tmp_path):
    bad = tmp_path / "bad.stl"
    bad.write_bytes(b"not an stl file at all")
    with pytest.raises(S.L.ASLError):
        S.readSTL(str(bad))
    with pytest.raises(S.L.ASLError):
        S.readSTL(str(tmp_path / "missing.stl"))
    with pytest.raises(S.L.ASLError, match="not supported"):
        S.readSurface(str(tmp_path / "x.obj"), 1.0)


@pytest.mark.parametrize("encoding,compress", [("ascii", False), ("binary", False), ("binary", True),
                                               ("appended", False), ("appended", True)])
def test_vtp_roundtrip(tmp_path, encoding, compress):
    sph = SO.icosphere(1.5, (0.5, -1.0, 2.0), subdiv=1)
    path = str(tmp_path / ("s_%s_%d.vtp" % (encoding, compress)))
    S.writeVTP(path, sph, encoding=encoding, compress=compress)
    got = S.readVTP(path)
    assert got.shape == sph.shape and np.array_equal(got, sph)


def test_vtp_polygons_become_triangle_fans(tmp_path):
    """A hand-written ascii file with one quad and one triangle sharing points."""
    path = tmp_path / "quad.vtp"
    path.write_text('<?xml version="1.0"?>\n<VTKFile type="PolyData" version="0.1" byte_order="LittleEndian">\n'
                    ' <PolyData><Piece NumberOfPoints="5" NumberOfPolys="2">\n'
                    '  <Points><DataArray type="Float32" NumberOfComponents="3" format="ascii">\n'
                    '   0 0 0  1 0 0  1 1 0  0 1 0  0 0 1</DataArray></Points>\n'
                    '  <Polys><DataArray type="Int32" Name="connectivity" format="ascii">0 1 2 3 0 1 4</DataArray>\n'
                    '   <DataArray type="Int32" Name="offsets" format="ascii">4 7</DataArray></Polys>\n'
                    ' </Piece></PolyData>\n</VTKFile>\n')
    got = S.readVTP(str(path))
    want = np.array([[[0, 0, 0], [1, 0, 0], [1, 1, 0]], [[0, 0, 0], [1, 1, 0], [0, 1, 0]],
                     [[0, 0, 0], [1, 0, 0], [0, 0, 1]]], dtype=np.float32)
    assert np.array_equal(got, want)
    bad = tmp_path / "img.vtp"
    bad.write_text('<?xml version="1.0"?><VTKFile type="ImageData"></VTKFile>')
    with pytest.raises(S.L.ASLError):
        S.readVTP(str(bad))
