"""GPU tests of ASL's C++ API (include/asl): programs written against ASL's
headers, compiled with g++ and linked against libaslb.so, run on the GPU and
match the FP32 oracle.

Tolerances: relative L2 of density and velocity over interior fluid cells
<= 1e-4 and drag within 1e-4 relative (the canonical channel after 1000
steps); the same bound on the pressure-driven D3Q15 channel after 200 steps.
"""
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from asl_b200 import geometry as G
from asl_b200 import writers as WR
from asl_b200.lbgk import Block

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def build(name: str, out: Path) -> Path:
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [cxx, "-std=c++17", "-O2", "-I", str(ROOT / "include" / "asl"), "-I", str(ROOT / "include"),
           str(ROOT / "examples" / "flow" / (name + ".cc")), "-L", str(ROOT / "asl_b200"), "-laslb",
           "-Wl,-rpath," + str(ROOT / "asl_b200"), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_canonical_channel_program_matches_oracle(gpu, cylinder_oracle, tmp_path):
    exe = build("channel_cylinder", tmp_path / "channel_cylinder")
    r = subprocess.run([str(exe), "--steps", "1000", "--output", str(tmp_path / "cc")], capture_output=True,
                       text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    drag = float(re.search(r"drag (\S+)", r.stdout).group(1))
    out = WR.read_vti(str(tmp_path / "cc_0.vti"))
    w = cylinder_oracle["workload"]
    # the program's map is the Python rasteriser's, bit for bit
    assert np.array_equal(out["map"], w.map[1:-1, 1:-1, 1:-1])
    fluid = w.map[1:-1, 1:-1, 1:-1] > 0
    assert rel(out["rho"][fluid], cylinder_oracle["rho"][1:-1, 1:-1, 1:-1][fluid]) <= 1e-4
    assert rel(out["v"][:, fluid], cylinder_oracle["u"][:, 1:-1, 1:-1, 1:-1][:, fluid]) <= 1e-4
    want = cylinder_oracle["force"][0]
    assert abs(drag - want) <= 1e-4 * abs(want), (drag, want)
    assert np.abs(out["force"]).max() > 0  # the force field was written


def test_pressure_channel_program_matches_oracle(gpu, oracle_mod, tmp_path):
    exe = build("pressure_channel", tmp_path / "pressure_channel")
    r = subprocess.run([str(exe), "--steps", "200", "--every", "100", "--output", str(tmp_path / "pc")],
                       capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "writes 2" in r.stdout
    size = (96, 32, 32)
    m = G.initData(Block(size, 1.0), G.generateDFCylinderInf(4.0, (0.0, 1.0, 0.0), (24.0, 0.0, 16.0)))
    o = oracle_mod.Oracle(size, 15, 4, 0.02)
    o.init_f(1.0, (0, 0, 0))
    ids = [o.bc_slice(2, 1, 1.02), o.bc_slice(2, 2, 0.98), o.bc_slice(0, 4 | 8 | 16 | 32), o.bc_map(10, m)]
    vis = o.bc_field(20, m)
    for n in range(1, 201):
        o.step(1)
        for i in ids:
            o.bc_execute(i)
        if n % 100 == 0:
            o.bc_execute(vis)
    out = WR.read_vti(str(tmp_path / "pc_1.vti"))
    assert np.array_equal(out["map"], m[1:-1, 1:-1, 1:-1])
    fluid = m[1:-1, 1:-1, 1:-1] > 0
    assert rel(out["rho"][fluid], o.get_rho()[1:-1, 1:-1, 1:-1][fluid]) <= 1e-4
    assert rel(out["v"][:, fluid], o.get_u()[:, 1:-1, 1:-1, 1:-1][:, fluid]) <= 1e-4
    # the visualisation condition set u on the guard cells
    guard = (m[1:-1, 1:-1, 1:-1] <= 0) & (m[1:-1, 1:-1, 1:-1] > -0.9999)
    assert guard.any()
    assert rel(out["v"][:, guard], o.get_u()[:, 1:-1, 1:-1, 1:-1][:, guard]) <= 1e-4


def test_read_surface_matches_python_reader(gpu, tmp_path):
    """readSurface (STL) through the C++ API: the block, spacing and offset
    overloads give the Python reader's maps and blocks bit for bit."""
    from asl_b200 import surface as S
    # a box and a tilted triangle fan, file coordinates (x, y, z)
    lo, hi = np.array([1.0, 0.5, -1.5]), np.array([4.0, 3.0, 2.5])
    v = np.array([[lo[0], lo[1], lo[2]], [hi[0], lo[1], lo[2]], [hi[0], hi[1], lo[2]], [lo[0], hi[1], lo[2]],
                  [lo[0], lo[1], hi[2]], [hi[0], lo[1], hi[2]], [hi[0], hi[1], hi[2]], [lo[0], hi[1], hi[2]]])
    faces = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (2, 3, 7), (2, 7, 6), (1, 2, 6),
             (1, 6, 5), (0, 4, 7), (0, 7, 3)]
    tri = np.array([[v[a], v[b], v[c]] for a, b, c in faces] + [[[0.0, 0.0, 0.0], [1.0, 0.2, 0.1], [0.3, 1.0, 0.4]]])
    path = tmp_path / "shape.stl"
    S.writeSTL(str(path), tri)
    src = ROOT / "tests" / "cpp" / "facade_surface.cc"
    cxx = shutil.which("g++") or "/usr/bin/g++"
    exe = tmp_path / "facade_surface"
    r = subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "include" / "asl"), "-I",
                        str(ROOT / "include"), str(src), "-L", str(ROOT / "asl_b200"), "-laslb",
                        "-Wl,-rpath," + str(ROOT / "asl_b200"), "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe), str(path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = {ln.split(" ", 1)[0]: ln.split(" ", 1)[1] for ln in r.stdout.splitlines()}
    want = {"block": S.readSurface(str(path), Block((24, 16, 12), 0.5, (-2.0, -1.0, 0.5))),
            "spacing": S.readSurface(str(path), 0.5),
            "offsets": S.readSurface(str(path), 0.5, 0.5, 0.25, 0.0, 1.0, 1.0, 0.5)}
    for k, m in want.items():
        f = got[k].split()
        b = m.getInternalBlock()
        assert tuple(int(x) for x in f[:3]) == tuple(b.size), k
        assert np.allclose([float(x) for x in f[3:6]], b.position, rtol=0, atol=1e-12), k
        assert float(f[6]) == b.dx, k
        vals = np.array([int(h, 16) for h in f[7:]], dtype=np.uint32).view(np.float32)
        assert np.array_equal(vals.reshape(m.shape), np.asarray(m, dtype=np.float32)), k
        assert np.asarray(m).min() < 0 < np.asarray(m).max()  # the surface lies inside the sampled grid
    assert got["error"] == "ASL ERROR: Reader: file format not supported"
