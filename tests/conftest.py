import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def gpu():
    """The CUDA library, loaded for GPU tests. Fails (does not skip) when the
    library or the device is missing: GPU tests must run on the native path."""
    import asl_b200._lib as L
    lib = L.load()
    L.check(lib.aslb_set_device(int(os.environ.get("ASLB_DEVICE", "0"))), "set_device")
    return lib


@pytest.fixture(scope="session")
def cylinder_oracle(oracle_mod):
    """The canonical cylinder channel (128x64x64, D3Q19, inlet 0.05, outlet
    pressure 1, no-slip walls and cylinder, nu 0.01) advanced 1000 steps by
    the FP32 oracle: its workload, density, velocity and surface force (about
    the cylinder axis point (32, 32, 31.5)). Computed once per session."""
    from asl_b200 import workloads as W
    w = W.channel_cylinder()
    o = oracle_mod.Oracle(w.size, 19, 4, w.nu)
    o.init_f(1.0, (0, 0, 0))
    ids = []
    for s in w.bcs:
        if s.kind == "map_noslip":
            ids.append(o.bc_map(10, w.map))
        else:
            ids.append(o.bc_slice(W.SLICE_KIND[s.kind], sum(W.WALL_BITS[x] for x in s.walls), s.p, s.u))
    for _ in range(w.steps):
        o.step(1)
        for i in ids:
            o.bc_execute(i)
    return {"workload": w, "rho": o.get_rho(), "u": o.get_u(), "force": o.force(w.map, r0=(32.0, 32.0, 31.5))}
