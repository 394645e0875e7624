"""TEST INFRASTRUCTURE, NOT PRODUCT CODE: ctypes wrapper of the CPU oracle.

The oracle (lbgk_oracle.cpp) restates ASL's LBGK path on the CPU. Only tests,
the smoke entry point and bench.py's CPU-baseline leg load it, as the checker.
Parity unpinned: the reference ships no golden vectors for this path; see the
header of lbgk_oracle.cpp for the known-answer pins.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "lbgk_oracle.cpp"
LIB = HERE / "liboracle.so"
# Portable x86-64 (AVX2) so the library built here also runs on the GPU box host.
CXXFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=c++17"]


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    # The system g++ ships the OpenMP runtime (libgomp).
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([cxx, *CXXFLAGS, str(SRC), "-o", str(tmp)], check=True)
    tmp.replace(LIB)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        vp, d, pd, pf = C.c_void_p, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_float)
        sig = {
            "orc_create": (vp, [C.c_int] * 5 + [d, C.c_int]),
            "orc_destroy": (None, [vp]),
            "orc_set_threads": (None, [C.c_int]),
            "orc_get_threads": (C.c_int, []),
            "orc_set_viscosity": (None, [vp, d]),
            "orc_set_body_force": (None, [vp, d, d, d]),
            "orc_set_omega": (None, [vp, d, d, d]),
            "orc_set_closure": (None, [vp, C.c_int, d]),
            "orc_set_position": (None, [vp, d, d, d, d]),
            "orc_init_f": (None, [vp, d, d, d, d]),
            "orc_init_f_fields": (None, [vp, pd, pd]),
            "orc_step": (None, [vp, C.c_int]),
            "orc_bc_slice": (C.c_int, [vp, C.c_int, C.c_int, d, d, d, d]),
            "orc_bc_map": (C.c_int, [vp, C.c_int, pf, d, pd, pd, pd]),
            "orc_bc_size": (C.c_long, [vp, C.c_int]),
            "orc_bc_execute": (None, [vp, C.c_int]),
            "orc_force": (None, [vp, pf, pf, pd, pd]),
            "orc_bc_deposition": (C.c_int, [vp, C.c_int, pf, d, d, d]),
            "orc_bc_map_cd": (C.c_int, [vp, C.c_int, pf, pf, d, pd, pd, pd]),
            "orc_bc_field": (C.c_int, [vp, C.c_int, pf, pd, pd, pd]),
            "orc_flux": (C.c_double, [vp, pf, pf]),
            "orc_size": (C.c_long, [vp]),
            "orc_get_f": (None, [vp, pd]),
            "orc_set_f": (None, [vp, pd]),
            "orc_get_rho": (None, [vp, pd]),
            "orc_get_u": (None, [vp, pd]),
            "orc_lattice": (None, [C.c_int, C.POINTER(C.c_int), pd, C.POINTER(C.c_int)]),
            "orc_sum": (d, [pd, C.c_long]),
            "orc_pack_spheres": (C.c_int, [C.c_int, C.c_int, C.c_int, d, d, d, C.c_ulonglong, C.c_int, C.c_int,
                                           C.c_int, pd, pd, C.POINTER(C.c_int)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def lattice(q: int):
    lib = load()
    c = (C.c_int * (3 * q))()
    w = (C.c_double * q)()
    inv = (C.c_int * q)()
    lib.orc_lattice(q, c, w, inv)
    return np.array(c[:]).reshape(q, 3), np.array(w[:]), np.array(inv[:])


def set_threads(n: int):
    load().orc_set_threads(int(n))


class Oracle:
    """One simulated domain. Same flag bits as the library: 1 no velocity, 2 no
    density, 4 incompressible, 8/16/32 periodic x/y/z."""

    def __init__(self, size, q=19, prec=4, nu=0.01, flags=0, position=(0.0, 0.0, 0.0), dx=1.0):
        self.lib = load()
        self.size = tuple(int(s) for s in size)
        self.q = q
        self.g = tuple(s + 2 for s in self.size)
        self.h = self.lib.orc_create(*self.size, q, prec, float(nu), int(flags))
        if not self.h:
            raise ValueError("oracle: bad arguments")
        self.lib.orc_set_position(self.h, *map(float, position), float(dx))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    def set_body_force(self, g):
        self.lib.orc_set_body_force(self.h, *map(float, g))

    def set_omega(self, w):
        self.lib.orc_set_omega(self.h, *map(float, w))

    def set_closure(self, mode, cs=0.17):
        self.lib.orc_set_closure(self.h, int(mode), float(cs))

    def set_viscosity(self, nu):
        self.lib.orc_set_viscosity(self.h, float(nu))

    def init_f(self, rho=1.0, u=(0.0, 0.0, 0.0)):
        self.lib.orc_init_f(self.h, float(rho), *map(float, u))

    def init_f_fields(self, rho, u):
        r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)
        uu = np.ascontiguousarray(u, dtype=np.float64)
        self.lib.orc_init_f_fields(self.h, _dp(r), _dp(uu))

    def step(self, n=1):
        self.lib.orc_step(self.h, int(n))

    def bc_slice(self, kind, wallmask, p=0.0, u=(0.0, 0.0, 0.0)) -> int:
        return self.lib.orc_bc_slice(self.h, int(kind), int(wallmask), float(p), *map(float, u))

    def bc_map(self, kind, m, p=0.0, u=(0.0, 0.0, 0.0), omega=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0),
               cdomain=None) -> int:
        mm = np.ascontiguousarray(m, dtype=np.float32)
        uu, om, ce = (np.asarray(v, dtype=np.float64) for v in (u, omega, center))
        if cdomain is not None:
            cd = np.ascontiguousarray(cdomain, dtype=np.float32)
            return self.lib.orc_bc_map_cd(self.h, int(kind), _fp(mm), _fp(cd), float(p), _dp(uu), _dp(om), _dp(ce))
        return self.lib.orc_bc_map(self.h, int(kind), _fp(mm), float(p), _dp(uu), _dp(om), _dp(ce))

    def bc_execute(self, bid):
        self.lib.orc_bc_execute(self.h, int(bid))

    def bc_size(self, bid) -> int:
        return int(self.lib.orc_bc_size(self.h, int(bid)))

    def bc_field(self, kind, m, u=(0.0, 0.0, 0.0), omega=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0)) -> int:
        mm = np.ascontiguousarray(m, dtype=np.float32)
        uu, om, ce = (np.asarray(v, dtype=np.float64) for v in (u, omega, center))
        return self.lib.orc_bc_field(self.h, int(kind), _fp(mm), _dp(uu), _dp(om), _dp(ce))

    def bc_deposition(self, kind, m, p0, lf, beta=0.0) -> int:
        mm = np.ascontiguousarray(m, dtype=np.float32)
        return self.lib.orc_bc_deposition(self.h, int(kind), _fp(mm), float(p0), float(lf), float(beta))

    def flux(self, m):
        """(flux field, FP64 total) of ComputeSurfaceFluxMap."""
        mm = np.ascontiguousarray(m, dtype=np.float32)
        fld = np.zeros(self.g, dtype=np.float32)
        tot = self.lib.orc_flux(self.h, _fp(mm), _fp(fld))
        return fld, float(tot)

    def force(self, m, r0=(0.0, 0.0, 0.0), field=False):
        mm = np.ascontiguousarray(m, dtype=np.float32)
        fld = np.zeros((3, *self.g), dtype=np.float32) if field else None
        out = np.zeros(6)
        self.lib.orc_force(self.h, _fp(mm), _fp(fld), _dp(np.asarray(r0, dtype=np.float64)), _dp(out))
        return (out, fld) if field else out

    def get_f(self):
        out = np.empty((self.q, *self.g))
        self.lib.orc_get_f(self.h, _dp(out))
        return out

    def set_f(self, f):
        self.lib.orc_set_f(self.h, _dp(np.ascontiguousarray(f, dtype=np.float64)))

    def get_rho(self):
        out = np.empty(self.g)
        self.lib.orc_get_rho(self.h, _dp(out))
        return out

    def get_u(self):
        out = np.empty((3, *self.g))
        self.lib.orc_get_u(self.h, _dp(out))
        return out


def reduction_sum(a) -> float:
    a = np.ascontiguousarray(a, dtype=np.float64)
    return float(load().orc_sum(_dp(a), a.size))


def pack_spheres(size, rmin: float, rmax: float, solid_fraction: float, seed: int, periodic_x: bool = True,
                 attempts: int = 400):
    """The porous channel's seeded sphere packing computed by the oracle
    library (the same spheres as the CUDA library's aslb_geom_pack_spheres),
    for CPU runs that must not load the product library. Returns
    (centers (n, 3), radii (n,))."""
    import math
    nx, ny, nz = (int(v) for v in size)
    cap = int(solid_fraction * nx * ny * nz / (4.0 / 3.0 * math.pi * rmin ** 3)) + 16
    centers = np.zeros((cap, 3))
    radii = np.zeros(cap)
    n = C.c_int(0)
    rc = load().orc_pack_spheres(nx, ny, nz, float(rmin), float(rmax), float(solid_fraction), int(seed),
                                 int(bool(periodic_x)), int(attempts), cap, _dp(centers), _dp(radii), C.byref(n))
    if rc != 0:
        raise ValueError("orc_pack_spheres: bad arguments")
    return centers[:n.value].copy(), radii[:n.value].copy()
