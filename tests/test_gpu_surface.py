"""GPU: surface distance maps (readSurface) against the oracle."""
import numpy as np
import pytest

from asl_b200 import lbgk as A
from asl_b200 import surface as S
from oracle import surface_oracle as SO

pytestmark = pytest.mark.gpu


def test_box_distance_and_interior(gpu):
    box = SO.box_mesh((2.3, 3.1, 1.7), (9.6, 7.2, 8.4))
    size, pos0, dx = (14, 12, 12), (0.1, 0.2, 0.3), 0.8
    band = 100.0  # the whole grid: every distance exact
    want = SO.distance_field(box, size, pos0, dx)
    got = S.surface_map(box, size, pos0, dx, 0.0, 1.0, band=band)
    assert np.abs(got - want).max() <= 1e-4
    inside = SO.inside_parity(box, size, pos0, dx)
    assert 0 < inside.sum() < inside.size
    got_s = S.surface_map(box, size, pos0, dx, 0.5, 2.0, solid_interior=True, band=band)
    assert np.abs(got_s - (np.where(inside, -want, want) - 0.5) / 2.0).max() <= 1e-4


def test_icosphere_band(gpu):
    sph = SO.icosphere(5.0, (8.2, 7.9, 8.1), subdiv=2)
    size, pos0, dx = (18, 17, 16), (0.0, 0.0, 0.0), 1.0
    want = SO.distance_field(sph, size, pos0, dx)
    got = S.surface_map(sph, size, pos0, dx, 0.0, 1.0, band=3.0)
    near = want <= 3.0
    assert np.abs(got[near] - want[near]).max() <= 1e-4
    assert np.all(got[~near] == np.float32(3.0))
    inside = SO.inside_parity(sph, size, pos0, dx)
    got_s = S.surface_map(sph, size, pos0, dx, 0.0, 1.0, solid_interior=True, band=3.0)
    assert np.array_equal(got_s < 0, inside & (want > 0))


def test_columns_through_shared_edges(gpu):
    """Columns that run exactly along the diagonals of the box's x faces (the
    edge two triangles share) count one crossing per face."""
    box = SO.box_mesh((1.5, 1.5, 1.5), (6.5, 6.5, 6.5))
    got = S.surface_map(box, (9, 9, 9), (0.0, 0.0, 0.0), 1.0, 0.0, 1.0, solid_interior=True, band=20.0)
    want = np.zeros((9, 9, 9), dtype=bool)
    want[2:7, 2:7, 2:7] = True
    assert np.array_equal(got < 0, want)


def test_read_surface_block_overload(gpu, tmp_path):
    """readSurface(file, block): block.size samples from block.position, ASL
    axes reversed from the file's (the file's X is ASL's z), offset 1.2 dx,
    scale 1.8 dx; the internal block is one cell smaller on every side."""
    # a bar long along the file's X axis
    bar = SO.box_mesh((2.0, 4.0, 5.0), (14.0, 8.0, 9.0))
    path = str(tmp_path / "bar.stl")
    S.writeSTL(path, bar)
    b = A.Block((14, 12, 18), 1.0, (0.5, 0.5, 0.5))
    m = S.readSurface(path, b)
    assert m.shape == (14, 12, 18) and m.dtype == np.float32
    ib = m.getInternalBlock()
    assert ib.size == (12, 10, 16) and ib.position == (1.5, 1.5, 1.5) and ib.dx == 1.0
    asl_bar = bar[..., ::-1]
    want = (SO.distance_field(asl_bar, b.size, b.position, 1.0) - 1.2) / 1.8
    near = want <= (4.0 - 1.2) / 1.8
    assert np.abs(m[near] - want[near]).max() <= 1e-4
    solid = m <= 0
    xs, ys, zs = np.nonzero(solid)
    assert zs.max() - zs.min() > xs.max() - xs.min()  # long along ASL z
    # usable as a map of the internal block
    lb = A.LBGK(ib, 0.05, A.d3q19())
    bc = A.generateBCNoSlip(lb, m)
    assert bc.num_links > 0


def test_read_surface_spacing_overloads(gpu, tmp_path):
    sph = SO.icosphere(3.0, (10.0, 20.0, 30.0), subdiv=1)
    path = str(tmp_path / "s.stl")
    S.writeSTL(path, sph, binary=False)
    m = S.readSurface(path, 0.5)
    ib = m.getInternalBlock()
    lo = sph.reshape(-1, 3)[:, ::-1].min(0) - 3.6 * 0.5
    assert np.allclose(np.asarray(ib.position) - 0.5, lo, atol=1e-5)
    assert m.min() < 0 < m.max()
    m2 = S.readSurface(path, 0.5, 0.5, 1.0, 0.0, 1.0, 2.0, 4.0)
    ext = sph.reshape(-1, 3)[:, ::-1].max(0) - sph.reshape(-1, 3)[:, ::-1].min(0)
    expect = [int(np.floor((ext[a] * (1 + f)) / 0.5)) + 1 for a, f in enumerate((1.5, 1.0, 6.0))]
    assert list(m2.shape) == expect


def test_read_surface_vtp_equals_stl(gpu, tmp_path):
    """readSurface gives the same map from the same surface in .stl and .vtp
    (compressed appended binary)."""
    sph = SO.icosphere(3.0, (8.0, 7.0, 6.0), subdiv=2)
    S.writeSTL(str(tmp_path / "s.stl"), sph)
    S.writeVTP(str(tmp_path / "s.vtp"), sph, encoding="appended", compress=True)
    b = A.Block((16, 14, 12), 1.0, (0.0, 0.0, 0.0))
    a = S.readSurface(str(tmp_path / "s.stl"), b)
    v = S.readSurface(str(tmp_path / "s.vtp"), b)
    assert np.array_equal(np.asarray(a), np.asarray(v))
    assert v.getInternalBlock().size == (14, 12, 10)
