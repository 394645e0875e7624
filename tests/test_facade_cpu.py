"""CPU tests of ASL's C++ API over the C ABI (include/asl): the example
programs compile and link against libaslb.so with the ASL header names, and
the host side of the facade (vectors, blocks, distance maps, parameters, the
VTK writer) behaves like ASL's and like the Python mirror."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from asl_b200 import geometry as G
from asl_b200 import writers as WR
from asl_b200.lbgk import Block

ROOT = Path(__file__).resolve().parents[1]


def cxx():
    c = shutil.which("g++") or "/usr/bin/g++"
    if not Path(c).exists():
        pytest.skip("no C++ compiler")
    return c


def build(src: Path, out: Path):
    cmd = [cxx(), "-std=c++17", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "include" / "asl"), "-I",
           str(ROOT / "include"), str(src), "-L", str(ROOT / "asl_b200"), "-laslb",
           "-Wl,-rpath," + str(ROOT / "asl_b200"), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.parametrize("name", ["channel_cylinder", "pressure_channel"])
def test_examples_compile_and_list_their_parameters(tmp_path, name):
    exe = build(ROOT / "examples" / "flow" / (name + ".cc"), tmp_path / name)
    r = subprocess.run([str(exe), "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "--steps" in r.stdout and "--device N" in r.stdout


def test_facade_host_side(tmp_path):
    exe = build(ROOT / "tests" / "cpp" / "facade_host.cc", tmp_path / "facade_host")
    r = subprocess.run([str(exe), "--size", "9 7 6", "--radius", "2.5", "--output", str(tmp_path / "fh")],
                       capture_output=True, text=True, timeout=60, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    lines = {ln.split(" ", 1)[0]: ln.split(" ", 1)[1] for ln in r.stdout.splitlines()}
    assert lines["params"] == "9 7 6 2.500 " + str(tmp_path / "fh")
    assert lines["dir"] == str(tmp_path.resolve()) + "/"  # no parameters file: the working directory
    assert lines["writes"] == "2"
    assert lines["error"] == "ASL ERROR: The inset is larger than the block size"
    # the FP32 map is bit for bit the Python rasteriser's (ASL's FP32 evaluation)
    block = Block((9, 7, 6), 0.5, (1.0, 2.0, 3.0))
    want = G.initData(block, G.normalize(G.generateDFCylinderInf(2.5, (0.0, 0.0, 1.0), (3.0, 4.0, 0.0)), 0.5))
    got = np.array([int(h, 16) for h in lines["map32"].split()], dtype=np.uint32).view(np.float32)
    assert np.array_equal(got.reshape(want.shape), want)
    assert float(lines["map64_vs_map32"]) < 1e-6
    # the writer: interior cells, ASL's axis and component order, read back
    for k in (0, 1):
        out = WR.read_vti(str(tmp_path / ("fh_%d.vti" % k)))
        assert np.array_equal(out["map"], want[1:-1, 1:-1, 1:-1])
        g = want.shape
        n = int(np.prod(g))
        vec = (np.arange(n, dtype=np.float64)[None] + 0.25 * np.arange(3)[:, None]).astype(np.float32)
        assert np.array_equal(out["vec"], vec.reshape(3, *g)[:, 1:-1, 1:-1, 1:-1])


def test_facade_rejects_unknown_and_missing_parameters(tmp_path):
    exe = build(ROOT / "tests" / "cpp" / "facade_host.cc", tmp_path / "facade_host")
    r = subprocess.run([str(exe), "--nosuch", "1"], capture_output=True, text=True, timeout=60, cwd=tmp_path)
    assert r.returncode != 0 and "unknown parameter" in r.stderr
    (tmp_path / "p.ini").write_text("# parameters\nradius = 1.5\nsize = 5 5 5\n")
    r = subprocess.run([str(exe), str(tmp_path / "p.ini"), "--output", str(tmp_path / "q")], capture_output=True,
                       text=True, timeout=60, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "params 5 5 5 1.500" in r.stdout


FLOW_EXAMPLES = ["flow", "flow2", "flow3", "flowRotatingCylinders", "locomotive", "locomotive_laminar",
                 "locomotive_stability", "bus_wind", "compressor"]


@pytest.mark.parametrize("name", FLOW_EXAMPLES)
def test_asl_flow_examples_compile_unchanged(tmp_path, name):
    """ASL's own LBGK example programs (examples/flow/*.cc of an ASL checkout
    named by ASL_REFERENCE_DIR) compile and link unchanged against these
    headers and libaslb.so. Skipped without a checkout."""
    import os
    ref = os.environ.get("ASL_REFERENCE_DIR")
    if not ref:
        pytest.skip("ASL_REFERENCE_DIR names no ASL checkout")
    src = Path(ref) / "examples" / "flow" / (name + ".cc")
    if not src.exists():
        pytest.skip("%s is not in the checkout" % src)
    cmd = [cxx(), "-std=c++17", "-O1", "-I", str(ROOT / "include" / "asl"), "-I", str(ROOT / "include"), str(src),
           "-L", str(ROOT / "asl_b200"), "-laslb", "-Wl,-rpath," + str(ROOT / "asl_b200"), "-o",
           str(tmp_path / name)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    h = subprocess.run([str(tmp_path / name), "--help"], capture_output=True, text=True, timeout=60)
    assert h.returncode == 0 and "--device N" in h.stdout
