"""CPU tests of the C ABI boundary: the library loads, exports every function
declared in include/aslb.h, and fails loudly (no CPU fallback) without a GPU."""
import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(aslb_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from asl_b200 import _lib as L
    if not L.LIB_PATH.exists():
        from asl_b200.build import build
        build()
    return L.load()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "aslb_lbgk_create" in names and "aslb_force_compute" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "asl_b200" / "libaslb.so")], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\s[TW]\s+(\w+)$", out, flags=re.M))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing


def test_python_binding_covers_header(lib):
    from asl_b200 import _lib as L
    assert set(declared_functions()) <= set(L.PROTOTYPES)


def test_library_is_sm100a_only():
    # The build emits sm_100a machine code only (no PTX for other targets).
    src = (ROOT / "asl_b200" / "build.py").read_text()
    assert "arch=compute_100a,code=sm_100a" in src


def test_no_gpu_fails_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from asl_b200 import lbgk as A
    with pytest.raises(A.L.ASLError):
        A.LBGK(A.Block((8, 8, 8)), 0.1, A.d3q19())


def test_argument_errors_without_gpu(lib):
    h = ctypes.c_void_p()
    assert lib.aslb_lbgk_create(0, 4, 4, 19, 0, 0.1, 0, ctypes.byref(h)) != 0
    assert b"sizes" in lib.aslb_last_error()
    assert lib.aslb_lbgk_create(4, 4, 4, 17, 0, 0.1, 0, ctypes.byref(h)) != 0
    assert b"q must be" in lib.aslb_last_error()
    assert lib.aslb_lbgk_create(4, 4, 4, 19, 0, -0.1, 0, ctypes.byref(h)) != 0
    assert lib.aslb_bc_execute(None) != 0
    assert lib.aslb_mlp_layout_bytes() > 0
