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
