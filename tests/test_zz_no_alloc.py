"""GPU tests of aslb_force_compute_noalloc, the surface-force entry point that
allocates nothing, for callers that cannot allocate device memory when they
ask for a force (a program whose allocator forbids new device allocations
after set-up, or a runtime that hands out all device memory up front). It
must give the same totals as aslb_force_compute, call after call, refuse
force-cell lists larger than its fixed scratch array, and refuse objects it
cannot serve without touching that array.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from asl_b200 import _lib as L
from asl_b200 import lbgk as A
from asl_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _noalloc(lib, force, r0):
    out = (C.c_double * 6)()
    L.check(lib.aslb_force_compute_noalloc(force.h, L.dvec(r0), out), "aslb_force_compute_noalloc")
    return np.array(out[:])


def test_noalloc_force_matches_allocating_entry_point(gpu):
    w = W.channel_cylinder(size=(64, 32, 24), radius=5.0, center=(20.0, 16.0), steps=0)
    lb, bcs = W.build_lbgk(w)
    force = A.generateComputeSurfaceForce(lb, w.map)
    r0 = (20.0, 16.0, 11.5)
    for steps in (30, 7):  # two calls in a row, each after the state changed
        lb.run(steps, bcs)
        want = force.execute(r0=r0)
        got = _noalloc(gpu, force, r0)
        assert np.allclose(got, want, rtol=1e-12, atol=1e-14), (got, want)
        again = _noalloc(gpu, force, r0)
        assert np.allclose(again, want, rtol=1e-12, atol=1e-14), (again, want)
    assert abs(want[0]) > 0


def test_noalloc_force_rejects_lists_beyond_its_scratch(gpu):
    w = W.porous_channel(size=(256, 128, 128), rmin=2.0, rmax=4.0, solid_fraction=0.35, steps=0)
    lb = A.LBGK(A.Block(w.size), w.nu, A.d3q19(), periodic=w.periodic)
    force = A.generateComputeSurfaceForce(lb, w.map)
    with pytest.raises(L.ASLError, match="scratch limit"):
        _noalloc(gpu, force, (0.0, 0.0, 0.0))
    assert np.isfinite(force.execute()).all()  # the allocating path still serves it


def test_noalloc_force_refuses_flux_objects_and_detached_forces(gpu):
    w = W.channel_cylinder(size=(32, 16, 16), radius=3.0, center=(10.0, 8.0), steps=0)
    lb, bcs = W.build_lbgk(w)
    lb.run(3, bcs)
    flux = C.c_void_p()
    L.check(gpu.aslb_flux_create(lb.h, w.map.ctypes.data_as(L._pf), C.byref(flux)), "aslb_flux_create")
    out = (C.c_double * 6)()
    assert gpu.aslb_force_compute_noalloc(flux, L.dvec((0.0, 0.0, 0.0)), out) == -1  # ASLB_ERR_ARG
    assert b"flux object" in gpu.aslb_last_error()
    gpu.aslb_flux_destroy(flux)
    assert gpu.aslb_force_compute_noalloc(None, L.dvec((0.0, 0.0, 0.0)), out) == -1
    # a force object whose domain was destroyed is detached: ASLB_ERR_STATE, no launch
    force = C.c_void_p()
    L.check(gpu.aslb_force_create(lb.h, w.map.ctypes.data_as(L._pf), C.byref(force)), "aslb_force_create")
    lb.close()
    assert gpu.aslb_force_compute_noalloc(force, L.dvec((0.0, 0.0, 0.0)), out) == -4  # ASLB_ERR_STATE
    assert b"destroyed" in gpu.aslb_last_error()
    gpu.aslb_force_destroy(force)
