"""CPU tests of the distance functions and the seeded workload geometry."""
import numpy as np

from asl_b200 import geometry as G
from asl_b200.lbgk import Block


def test_sphere_sign_and_normalize():
    b = Block((10, 10, 10))
    m = G.initData(b, G.normalize(G.generateDFSphere(3.0, (4.5, 4.5, 4.5)), 1.0))
    assert m.dtype == np.float32 and m.shape == (12, 12, 12)
    assert m[1 + 4, 1 + 4, 1 + 4] < 0  # inside (distance ~ -2.1)
    assert m[1, 1, 1] == 1.0  # far outside, clipped
    assert m.min() >= -1.0 and m.max() <= 1.0
    # position of ghosted cell g is block.position + (g - 1) dx (aslGeomInc.cxx:192)
    raw = G.initData(b, G.generateDFSphere(3.0, (4.5, 4.5, 4.5)))
    assert abs(raw[5, 5, 5] - (np.sqrt(3 * 0.25) - 3.0)) < 1e-6


def test_union_intersection_inversion():
    b = Block((8, 8, 8))
    s1 = G.generateDFSphere(2.0, (2, 2, 2))
    s2 = G.generateDFSphere(2.0, (5, 5, 5))
    u = G.initData(b, s1 | s2)
    i = G.initData(b, s1 & s2)
    n = G.initData(b, -s1)
    a1, a2 = G.initData(b, s1), G.initData(b, s2)
    assert np.array_equal(u, np.minimum(a1, a2))
    assert np.array_equal(i, np.maximum(a1, a2))
    assert np.array_equal(n, -a1)


def test_cylinder_and_box():
    b = Block((16, 16, 8))
    cyl = G.initData(b, G.generateDFCylinderInf(3.0, (0, 0, 1), (8.0, 8.0, 0.0)))
    assert cyl[9, 9, 0] < 0 and cyl[9, 9, 9] < 0  # infinite along z
    fin = G.initData(b, G.generateDFCylinder(3.0, (0, 0, 4.0), (8.0, 8.0, 3.5)))
    assert fin[9, 9, 4] < 0 and fin[9, 9, 8] > 0
    box = G.initData(b, G.generateDFBox((8.0, 8.0, 4.0), (2.0, 3.0, 1.0)))
    assert box[9, 9, 5] < 0 and box[9, 11, 5] < 0 and box[9, 12, 5] == 0 and box[9, 13, 5] > 0


def test_sphere_pack_is_seeded_and_non_overlapping():
    p1 = G.pack_spheres((96, 48, 48), 4, 8, 0.3, seed=5)
    p2 = G.pack_spheres((96, 48, 48), 4, 8, 0.3, seed=5)
    assert np.array_equal(p1.centers, p2.centers)
    c, r = p1.centers, p1.radii
    d = c[:, None, :] - c[None, :, :]
    d[..., 0] -= 96 * np.round(d[..., 0] / 96)
    dist = np.sqrt((d ** 2).sum(-1))
    np.fill_diagonal(dist, np.inf)
    assert (dist >= (r[:, None] + r[None, :]) - 1e-9).all()
    assert (c[:, 1] >= r - 1e-9).all() and (c[:, 1] <= 47 - r + 1e-9).all()
    vol = (4 / 3 * np.pi * r ** 3).sum() / (96 * 48 * 48)
    assert vol >= 0.3


def _assert_no_overlap(c, r, nx):
    d = c[:, None, :] - c[None, :, :]
    d[..., 0] -= nx * np.round(d[..., 0] / nx)
    dist = np.sqrt((d ** 2).sum(-1))
    np.fill_diagonal(dist, np.inf)
    assert (dist >= (r[:, None] + r[None, :]) - 1e-9).all()


def test_sphere_pack_no_overlap_across_the_periodic_seam():
    # 100 is not a multiple of the 2 rmax = 16 bucket width: spheres near
    # x = 0 and x = 100 are neighbours across the seam
    for seed in range(6):
        p = G.pack_spheres((100, 40, 40), 4, 8, 0.35, seed=seed)
        _assert_no_overlap(p.centers, p.radii, 100)


def test_sphere_pack_matches_the_oracle_packer():
    """The CPU benchmark runs build the porous channel with the oracle's
    packer (no CUDA library): it must give the library's spheres bit for bit."""
    from oracle import oracle as O
    for size, per, seed in [((100, 40, 40), True, 1), ((96, 48, 48), True, 5), ((90, 40, 50), False, 2),
                            ((256, 128, 128), True, 20261205)]:
        p = G.pack_spheres(size, 4, 12, 0.4, seed=seed, periodic_x=per)
        c, r = O.pack_spheres(size, 4, 12, 0.4, seed, per)
        assert len(r) > 0
        assert np.array_equal(p.centers, c) and np.array_equal(p.radii, r)


def test_rasterized_spheres_match_direct_union():
    b = Block((40, 20, 20))
    p = G.pack_spheres((40, 20, 20), 2, 4, 0.2, seed=3)
    fast = G.rasterize_spheres(b, p, periodic_x=True)
    df = None
    for c, r in zip(p.centers, p.radii):
        for sx in (-40, 0, 40):
            s = G.generateDFSphere(r, (c[0] + sx, c[1], c[2]))
            df = s if df is None else (df | s)
    direct = G.initData(b, G.normalize(df, 1.0))
    assert np.abs(fast - direct).max() < 1e-5


def test_rasterized_union_matches_direct_union():
    b = Block((30, 20, 16))
    shapes = [(G.generateDFBox((8.0, 6.0, 3.5), (3.0, 2.0, 4.0)), (5.0, 4.0, -0.5), (11.0, 8.0, 7.5)),
              (G.generateDFCylinder(2.5, (0.0, 0.0, 6.0), (20.0, 12.0, 2.5)), (17.5, 9.5, -0.5), (22.5, 14.5, 5.5))]
    fast = G.rasterize_union(b, shapes)
    direct = G.initData(b, G.normalize(shapes[0][0] | shapes[1][0], 1.0))
    assert np.abs(fast - direct).max() < 1e-6


def test_vehicle_workload_is_seeded_and_on_the_floor():
    from asl_b200 import workloads as W
    a = W.vehicle_d3q27(size=(96, 48, 48))
    b = W.vehicle_d3q27(size=(96, 48, 48))
    assert np.array_equal(a.map, b.map) and a.q == 27
    solid = a.map[1:-1, 1:-1, 1:-1] <= 0
    assert 0.002 < solid.mean() < 0.1
    # every obstacle stands on the floor: solid cells in the first layer, none at the top
    assert solid[:, :, 0].any() and not solid[:, :, -1].any()
    assert [s.kind for s in a.bcs] == ["velocity", "pressure", "map_noslip"]


def test_union_and_intersection_start_from_none():
    """ASL's operators take an uninitialised operand as the identity."""
    s = G.generateDFSphere(2.0, (3.0, 3.0, 3.0))
    block = Block((6, 6, 6), 1.0)
    acc = None
    acc = acc | s
    assert acc is s and (s | None) is s and (None & s) is s and (s & None) is s
    assert np.array_equal(G.initData(block, acc), G.initData(block, s))
