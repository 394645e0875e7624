"""Python mirror of ASL's LBGK API over the C ABI of libaslb.so.

Names and argument meaning follow the reference's C++ interface
(src/num/aslLBGK.h, src/num/aslLBGKBC.h, src/num/aslNumMethod.h of
AvtechScientific/ASL) so that a script reads like an ASL example program:

    block = Block((128, 64, 64), 1.0)
    lbgk = LBGK(block, 0.01, d3q19())
    lbgk.init()
    LBGKUtilities(lbgk).initF((0.0, 0.0, 0.0))
    bc = [generateBCConstantVelocity(lbgk, (0.05, 0, 0), [X0]), ...]
    initAll(bc)
    for n in range(1000):
        lbgk.execute(); executeAll(bc)

Fields come back as numpy arrays over the ghosted block, shape
(nx+2, ny+2, nz+2) (vector fields: (3, nx+2, ny+2, nz+2)), in ASL's
flattening order (z fastest).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from enum import IntEnum
from typing import Iterable, Sequence

import numpy as np

from . import _lib as L


class SlicesNames(IntEnum):
    """Walls of the box (src/num/aslBCond.h:309)."""
    X0 = 0
    XE = 1
    Y0 = 2
    YE = 3
    Z0 = 4
    ZE = 5


X0, XE, Y0, YE, Z0, ZE = (SlicesNames(i) for i in range(6))


@dataclass(frozen=True)
class VectorTemplate:
    """Velocity set (src/math/aslTemplates.h): q directions in ASL's order."""
    q: int

    @property
    def vectors(self) -> np.ndarray:
        return lattice_vectors(self.q)

    @property
    def quasiparticlesCoefs(self) -> np.ndarray:
        return lattice_weights(self.q)


def lattice_vectors(q: int) -> np.ndarray:
    v27 = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (-1, 0, 0), (0, -1, 0), (0, 0, -1),
           (1, 1, 0), (1, -1, 0), (-1, -1, 0), (-1, 1, 0), (0, 1, 1), (0, 1, -1), (0, -1, -1),
           (0, -1, 1), (1, 0, 1), (1, 0, -1), (-1, 0, -1), (-1, 0, 1), (1, 1, 1), (1, 1, -1),
           (1, -1, 1), (1, -1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1)]
    if q == 15:
        return np.array(v27[:7] + v27[19:], dtype=np.int64)
    return np.array(v27[:q], dtype=np.int64)


def lattice_weights(q: int) -> np.ndarray:
    n2 = (lattice_vectors(q) ** 2).sum(1)
    table = {15: {0: 2 / 9, 1: 1 / 9, 3: 1 / 72},
             19: {0: 1 / 3, 1: 1 / 18, 2: 1 / 36},
             27: {0: 8 / 27, 1: 2 / 27, 2: 1 / 54, 3: 1 / 216}}[q]
    return np.array([table[int(a)] for a in n2])


def d3q15() -> VectorTemplate:
    return VectorTemplate(15)


def d3q19() -> VectorTemplate:
    return VectorTemplate(19)


def d3q27() -> VectorTemplate:
    return VectorTemplate(27)


class Block:
    """Simulation grid (src/data/aslBlocks.h:56-88): interior size, spacing and
    the physical position of interior cell (0, 0, 0)."""

    def __init__(self, size: Sequence[int], dx: float = 1.0, position: Sequence[float] = (0.0, 0.0, 0.0)):
        self.size = tuple(int(s) for s in size)
        if len(self.size) != 3 or min(self.size) < 1:
            raise L.ASLError("ASL ERROR: Block: three positive sizes required")
        self.dx = float(dx)
        self.position = tuple(float(p) for p in position)

    def getSize(self):
        return self.size

    @property
    def ghosted(self):
        return tuple(s + 2 for s in self.size)

    def c2i(self, c):
        """Flattened index of ghosted coordinates (z fastest)."""
        gx, gy, gz = self.ghosted
        return (c[0] * gy + c[1]) * gz + c[2]

    def positions(self):
        """Physical coordinates of every ghosted cell, shape (3, gx, gy, gz)."""
        axes = [self.position[a] + (np.arange(self.ghosted[a]) - 1) * self.dx for a in range(3)]
        return np.stack(np.meshgrid(*axes, indexing="ij"))


_STORAGE = {"f32": L.F32, "f16": L.F16, "f64": L.F64, np.float32: L.F32, np.float64: L.F64}


class LBGK:
    """Fused stream-collide LBGK (src/num/aslLBGK.h:77-131).

    ``storage`` picks the population format: "f32" (ASL with FlT=float), "f64"
    (FlT=double) or "f16" (shifted FP16 deviations, FP32 arithmetic).
    ``periodic`` (x, y, z), ``body_force`` and ``packed_rows`` (z rows back to
    back, for short rows) are extensions without an ASL analogue."""

    closure = L.CLOSURE_NONE

    def __init__(self, block: Block, nu: float, vt: VectorTemplate, compVel: bool = True, compRho: bool = True,
                 storage="f32", periodic=(False, False, False), body_force=None, packed_rows: bool = False):
        self.lib = L.load()
        self.block = block
        self.vectorTemplate = vt
        st = _STORAGE[storage]
        flags = (0 if compVel else L.NO_VELOCITY) | (0 if compRho else L.NO_RHO)
        if packed_rows:
            flags |= L.PACKED_ROWS
        for a, p in enumerate(periodic):
            if p:
                flags |= (L.PERIODIC_X, L.PERIODIC_Y, L.PERIODIC_Z)[a]
        self.periodic = tuple(bool(p) for p in periodic)
        self.storage = storage
        h = C.c_void_p()
        nx, ny, nz = block.size
        L.check(self.lib.aslb_lbgk_create(nx, ny, nz, vt.q, st, float(nu), flags, C.byref(h)), "LBGK")
        self.h = h
        L.check(self.lib.aslb_lbgk_set_position(h, L.dvec(block.position), block.dx), "LBGK")
        if body_force is not None:
            self.setBodyForce(body_force)
        self._inited = False

    # lifecycle (NumMethod: src/num/aslNumMethod.h:34-77)
    def init(self):
        if self.closure != L.CLOSURE_NONE:
            L.check(self.lib.aslb_lbgk_set_closure(self.h, self.closure, getattr(self, "cs", 0.17)), "LBGK::init")
        self._inited = True

    def execute(self, nsteps: int = 1):
        L.check(self.lib.aslb_lbgk_step(self.h, int(nsteps)), "LBGK::execute")

    def run(self, nsteps: int, bcs: Sequence["BC"] = (), use_graph: bool = True):
        """`for n: execute(); executeAll(bcs)` in one call (graph replay)."""
        arr = (C.c_void_p * max(1, len(bcs)))(*[b.h for b in bcs])
        L.check(self.lib.aslb_lbgk_run(self.h, int(nsteps), arr, len(bcs), 1 if use_graph else 0), "LBGK::run")

    def sync(self):
        L.check(self.lib.aslb_lbgk_sync(self.h), "LBGK::sync")

    def setKernel(self, variant: int):
        """0: direct loads, two cells per thread where available (default);
        1: TMA-staged persistent kernel; 2: direct loads, one cell per thread."""
        L.check(self.lib.aslb_lbgk_set_kernel(self.h, int(variant)), "LBGK::setKernel")

    @property
    def kernel(self) -> int:
        return int(self.lib.aslb_lbgk_get_kernel(self.h))

    @property
    def steps(self) -> int:
        return int(self.lib.aslb_lbgk_steps(self.h))

    @property
    def stream(self) -> int:
        return int(self.lib.aslb_lbgk_stream(self.h) or 0)

    # parameters
    def setViscosity(self, nu: float):
        L.check(self.lib.aslb_lbgk_set_viscosity(self.h, float(nu)), "LBGK::setViscosity")

    def getViscosity(self) -> float:
        return float(self.lib.aslb_lbgk_get_viscosity(self.h))

    def setOmega(self, w):
        L.check(self.lib.aslb_lbgk_set_omega(self.h, L.dvec(w)), "LBGK::setOmega")

    def setCompressible(self, flag: bool = True):
        L.check(self.lib.aslb_lbgk_set_compressible(self.h, 1 if flag else 0), "LBGK::setCompressible")

    def setBodyForce(self, g):
        L.check(self.lib.aslb_lbgk_set_body_force(self.h, L.dvec(g)), "LBGK::setBodyForce")

    def setMacroOutput(self, compVel: bool, compRho: bool):
        L.check(self.lib.aslb_lbgk_set_macro_output(self.h, int(compVel), int(compRho)), "LBGK")

    def requestMacro(self):
        L.check(self.lib.aslb_lbgk_request_macro(self.h), "LBGK")

    def setClosure(self, closure: int, cs: float = 0.17):
        L.check(self.lib.aslb_lbgk_set_closure(self.h, int(closure), float(cs)), "LBGK::setClosure")

    def setFP16Scale(self, scale: float):
        L.check(self.lib.aslb_lbgk_set_fp16_scale(self.h, float(scale)), "LBGK")

    def setMLP(self, blob: bytes):
        buf = C.create_string_buffer(bytes(blob), len(blob))
        L.check(self.lib.aslb_lbgk_set_mlp(self.h, C.cast(buf, C.c_void_p), len(blob)), "LBGK::setMLP")

    def setMLPPeriod(self, steps: int):
        """Steps between two evaluations of the closure network (default 32)."""
        L.check(self.lib.aslb_lbgk_set_mlp_period(self.h, int(steps)), "LBGK::setMLPPeriod")

    def closureFeatures(self, out_dev_ptr: int):
        """Write the nine raw closure features of every interior cell to device
        memory at ``out_dev_ptr`` (9 x cells floats, cells x-major, z fastest)."""
        L.check(self.lib.aslb_lbgk_closure_features(self.h, C.c_void_p(int(out_dev_ptr))), "LBGK::closureFeatures")

    def getCs2(self, dtype=np.float64) -> np.ndarray:
        """The learned closure's Cs^2 field the next step uses (ghosted layout)."""
        return self._read(L.FIELD_CS2, 1, dtype)[0]

    def getVectorTemplate(self) -> VectorTemplate:
        return self.vectorTemplate

    # data (getRho / getVelocity / getF + acl::map)
    def _read(self, field: int, ncomp: int, dtype=np.float64) -> np.ndarray:
        gx, gy, gz = self.block.ghosted
        out = np.empty((ncomp, gx, gy, gz), dtype=dtype)
        code = L.F64 if dtype == np.float64 else L.F32
        L.check(self.lib.aslb_lbgk_read(self.h, field, code, out.ctypes.data_as(C.c_void_p)), "LBGK::read")
        return out

    def getRho(self, dtype=np.float64) -> np.ndarray:
        return self._read(L.FIELD_RHO, 1, dtype)[0]

    def getVelocity(self, dtype=np.float64) -> np.ndarray:
        return self._read(L.FIELD_VELOCITY, 3, dtype)

    def getF(self, dtype=np.float64) -> np.ndarray:
        return self._read(L.FIELD_F, self.vectorTemplate.q, dtype)

    def setF(self, f: np.ndarray):
        f = np.ascontiguousarray(f, dtype=np.float64)
        if f.shape != (self.vectorTemplate.q, *self.block.ghosted):
            raise L.ASLError("ASL ERROR: setF: wrong shape")
        L.check(self.lib.aslb_lbgk_write(self.h, L.FIELD_F, L.F64, f.ctypes.data_as(C.c_void_p)), "LBGK::setF")

    def saveState(self):
        """Restart dump: (population array bytes as stored, meta = [steps,
        parity, fused links active, storage])."""
        n = int(self.lib.aslb_lbgk_state_bytes(self.h))
        buf = np.empty(n, dtype=np.uint8)
        meta = (C.c_longlong * 4)()
        L.check(self.lib.aslb_lbgk_save_state(self.h, buf.ctypes.data_as(C.c_void_p), n, meta), "LBGK::saveState")
        return buf, np.array(meta[:], dtype=np.int64)

    def loadState(self, data: np.ndarray, meta):
        data = np.ascontiguousarray(data, dtype=np.uint8)
        m = (C.c_longlong * 4)(*[int(v) for v in meta])
        L.check(self.lib.aslb_lbgk_load_state(self.h, data.ctypes.data_as(C.c_void_p), data.nbytes, m),
                "LBGK::loadState")

    def watchdog(self) -> dict:
        """Largest |u|, smallest rho and number of non-finite cells (FP64)."""
        out = (C.c_double * 3)()
        L.check(self.lib.aslb_lbgk_watchdog(self.h, out), "LBGK::watchdog")
        return {"max_u": out[0], "min_rho": out[1], "nonfinite": int(out[2])}

    def moments(self) -> np.ndarray:
        out = (C.c_double * 4)()
        L.check(self.lib.aslb_lbgk_moments(self.h, out), "LBGK::moments")
        return np.array(out[:])

    def close(self):
        if getattr(self, "h", None):
            self.lib.aslb_lbgk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LBGKTurbulence(LBGK):
    """asl::LBGKTurbulence (src/num/aslLBGK.h:163-171) with its limiter
    evaluated on a defined f_eq (the reference reads f_eq before assigning it)."""
    closure = L.CLOSURE_ASL_INTENT


class LBGKSmagorinsky(LBGK):
    """Extension: Smagorinsky closure (Hou et al. 1996), constant ``cs``."""
    closure = L.CLOSURE_SMAGORINSKY

    def __init__(self, *args, cs: float = 0.17, **kw):
        self.cs = float(cs)
        super().__init__(*args, **kw)


class LBGKUtilities:
    """src/num/aslLBGK.h:137-159: initF(vel) or initF(rho, vel); rho and vel
    are constants or ghosted-block arrays."""

    def __init__(self, lbgk: LBGK):
        self.num = lbgk

    def initF(self, a, b=None):
        rho, vel = (1.0, a) if b is None else (a, b)
        lib = self.num.lib
        if np.ndim(vel) == 1 and np.ndim(rho) == 0:
            L.check(lib.aslb_lbgk_init_f(self.num.h, float(rho), L.dvec(vel)), "LBGKUtilities::initF")
            return
        g = self.num.block.ghosted
        v = np.asarray(vel, dtype=np.float64)
        if v.ndim == 1:
            v = v.reshape(3, 1, 1, 1)
        u = np.ascontiguousarray(np.broadcast_to(v, (3, *g)))
        r = None if np.ndim(rho) == 0 and float(rho) == 1.0 else np.ascontiguousarray(
            np.broadcast_to(np.asarray(rho, dtype=np.float64), g))
        L.check(lib.aslb_lbgk_init_f_fields(self.num.h, None if r is None else r.ctypes.data_as(L._pd),
                                            u.ctypes.data_as(L._pd)), "LBGKUtilities::initF")

    # Declared but never defined by the reference (src/num/aslLBGK.h:153-155):
    # the density / velocity fields from the populations as they stand.
    def computeRho(self):
        L.check(self.num.lib.aslb_lbgk_compute_macro(self.num.h, 1, 0), "LBGKUtilities::computeRho")

    def computeVelocity(self):
        L.check(self.num.lib.aslb_lbgk_compute_macro(self.num.h, 0, 1), "LBGKUtilities::computeVelocity")

    def computeRhoVelocity(self):
        L.check(self.num.lib.aslb_lbgk_compute_macro(self.num.h, 1, 1), "LBGKUtilities::computeRhoVelocity")


# ---- boundary conditions -----------------------------------------------------

class BC:
    """A boundary condition bound to one LBGK (BCond / BCondWithMap)."""

    def __init__(self, lbgk: LBGK, h: C.c_void_p):
        self.num = lbgk
        self.h = h

    def init(self):
        pass

    def execute(self):
        L.check(self.num.lib.aslb_bc_execute(self.h), "BCond::execute")

    @property
    def num_links(self) -> int:
        return int(self.num.lib.aslb_bc_num_links(self.h))

    @property
    def kernels(self) -> int:
        """Kernel launches per execute()."""
        return int(self.num.lib.aslb_bc_kernels(self.h))

    def fuse(self):
        """Fold this no-slip condition into the stream-collide kernel
        (extension): bounce-back happens inline, results are unchanged."""
        L.check(self.num.lib.aslb_bc_fuse(self.h), "BCNoSlip::fuse")

    @property
    def fused(self) -> bool:
        return bool(self.num.lib.aslb_bc_is_fused(self.h))

    def __del__(self):
        try:
            if self.h:
                self.num.lib.aslb_bc_destroy(self.h)
                self.h = None
        except Exception:
            pass


def _wallmask(slices: Iterable[SlicesNames]) -> int:
    m = 0
    for s in slices:
        m |= 1 << int(s)
    return m


def _is_map(x) -> bool:
    return isinstance(x, np.ndarray)


def _map_array(lbgk: LBGK, m: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(m, dtype=np.float32)
    if m.shape != lbgk.block.ghosted:
        raise L.ASLError(f"ASL ERROR: map must cover the ghosted block {lbgk.block.ghosted}, got {m.shape}")
    return m


def _slice_bc(lbgk: LBGK, kind: int, slices, p: float = 0.0, u=(0.0, 0.0, 0.0)) -> BC:
    h = C.c_void_p()
    L.check(lbgk.lib.aslb_bc_slice_create(lbgk.h, kind, _wallmask(slices), float(p), L.dvec(u), C.byref(h)),
            "generateBC")
    return BC(lbgk, h)


def _map_bc(lbgk: LBGK, kind: int, m, p=0.0, u=(0.0, 0.0, 0.0), omega=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0),
            cdomain=None) -> BC:
    arr = _map_array(lbgk, m)
    cd = None if cdomain is None else _map_array(lbgk, cdomain)
    h = C.c_void_p()
    L.check(lbgk.lib.aslb_bc_map_create_cd(lbgk.h, kind, arr.ctypes.data_as(L._pf),
                                           None if cd is None else cd.ctypes.data_as(L._pf), float(p), L.dvec(u),
                                           L.dvec(omega), L.dvec(center), C.byref(h)), "generateBC")
    return BC(lbgk, h)


def generateBCNoSlip(lbgk: LBGK, where) -> BC:
    """Bounce-back on walls (src/num/aslLBGKBC.cxx:745-751) or on a map (:801-805)."""
    if _is_map(where):
        return _map_bc(lbgk, L.BC_MAP_NOSLIP, where)
    return _slice_bc(lbgk, L.BC_NOSLIP, where)


def generateBCConstantVelocity(lbgk: LBGK, v, slices) -> BC:
    return _slice_bc(lbgk, L.BC_VELOCITY, slices, u=v)


def generateBCConstantPressure(lbgk: LBGK, p: float, where) -> BC:
    if _is_map(where):
        return _map_bc(lbgk, L.BC_MAP_PRESSURE_VELOCITY, where, p=p)
    return _slice_bc(lbgk, L.BC_PRESSURE, where, p=p)


def generateBCConstantPressureVelocity(lbgk: LBGK, p: float, v, where) -> BC:
    if _is_map(where):
        return _map_bc(lbgk, L.BC_MAP_PRESSURE_VELOCITY, where, p=p, u=v)
    return _slice_bc(lbgk, L.BC_PRESSURE_VELOCITY, where, p=p, u=v)


@dataclass
class PFConstant:
    """generatePFConstant(v)."""
    value: tuple


@dataclass
class PFRotationField:
    """generatePFRotationField(omega, center): u = omega x (r - center)."""
    omega: tuple
    center: tuple


def generatePFConstant(v) -> PFConstant:
    return PFConstant(tuple(float(a) for a in v))


def generatePFRotationField(omega, center) -> PFRotationField:
    return PFRotationField(tuple(float(a) for a in omega), tuple(float(a) for a in center))


def generateBCVelocity(lbgk: LBGK, velocity, m, computationalDomain=None) -> BC:
    """BCVelocityMap (src/num/aslLBGKBC.cxx:262-354) with a constant or rotation
    field; with ``computationalDomain`` only neighbours where that map is
    positive are fluid ends (the four-argument overload, :837-844)."""
    if isinstance(velocity, PFRotationField):
        return _map_bc(lbgk, L.BC_MAP_VELOCITY_ROTATION, m, omega=velocity.omega, center=velocity.center,
                       cdomain=computationalDomain)
    if isinstance(velocity, PFConstant):
        velocity = velocity.value
    return _map_bc(lbgk, L.BC_MAP_VELOCITY, m, u=velocity, cdomain=computationalDomain)


def _field_bc(lbgk: LBGK, kind: int, m, u=(0.0, 0.0, 0.0), omega=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0)) -> BC:
    arr = _map_array(lbgk, m)
    h = C.c_void_p()
    L.check(lbgk.lib.aslb_bc_field_create(lbgk.h, kind, arr.ctypes.data_as(L._pf), L.dvec(u), L.dvec(omega),
                                          L.dvec(center), C.byref(h)), "generateBC")
    return BC(lbgk, h)


def generateBCNoSlipVel(lbgk: LBGK, m) -> BC:
    """Velocity output zero at the map surface, for visualisation
    (src/num/aslLBGKBC.cxx:808-816: BCConstantValueMiddlePointMap on u)."""
    return _field_bc(lbgk, L.BC_FIELD_NOSLIP_VEL, m)


def generateBCNoSlipRho(lbgk: LBGK, m) -> BC:
    """Zero normal gradient of the density output at the map surface
    (src/num/aslLBGKBC.cxx:819-827: BCConstantGradientMap on rho)."""
    return _field_bc(lbgk, L.BC_FIELD_NOSLIP_RHO, m)


def generateBCVelocityVel(lbgk: LBGK, velocity, m) -> BC:
    """Velocity output set to a position function on the map's guard cells
    (src/num/aslLBGKBC.cxx:847-852: BCValuePFMap on u)."""
    if isinstance(velocity, PFRotationField):
        return _field_bc(lbgk, L.BC_FIELD_VELOCITY_VEL_ROTATION, m, omega=velocity.omega, center=velocity.center)
    if isinstance(velocity, PFConstant):
        velocity = velocity.value
    return _field_bc(lbgk, L.BC_FIELD_VELOCITY_VEL, m, u=velocity)


def _deposition_bc(lbgk: LBGK, kind: int, m, p0: float, lf: float, beta: float) -> BC:
    arr = _map_array(lbgk, m)
    h = C.c_void_p()
    L.check(lbgk.lib.aslb_bc_deposition_create(lbgk.h, kind, arr.ctypes.data_as(L._pf), float(p0), float(lf),
                                               float(beta), C.byref(h)), "generateBCDeposition")
    return BC(lbgk, h)


def generateBCTransportLimitedDeposition(lbgk: LBGK, p0: float, limitingFactor: float, m) -> BC:
    """BCTransportLimitedDepositionMap (src/num/aslLBGKBC.cxx:440-506, 878-888)."""
    return _deposition_bc(lbgk, L.BC_MAP_TRANSPORT_DEPOSITION, m, p0, limitingFactor, 0.0)


def generateBCKineticsLimitedDeposition(lbgk: LBGK, p0: float, limitingFactor: float, beta: float, m) -> BC:
    """BCKineticsLimitedDepositionMap (src/num/aslLBGKBC.cxx:508-575, 891-903);
    the arguments in the order of the definition (the header names them
    beta, p0, limitingFactor, but binds them positionally as here)."""
    return _deposition_bc(lbgk, L.BC_MAP_KINETICS_DEPOSITION, m, p0, limitingFactor, beta)


class ComputeSurfaceFlux:
    """ComputeSurfaceFluxMap (src/num/aslLBGKBC.cxx:623-665): ``execute()``
    returns the flux field (ghosted, FP32; cells off the surface 0) and its
    FP64 total."""

    def __init__(self, lbgk: LBGK, m: np.ndarray):
        self.num = lbgk
        arr = _map_array(lbgk, m)
        h = C.c_void_p()
        L.check(lbgk.lib.aslb_flux_create(lbgk.h, arr.ctypes.data_as(L._pf), C.byref(h)), "ComputeSurfaceFlux")
        self.h = h

    def init(self):
        pass

    def execute(self):
        fld = np.zeros(self.num.block.ghosted, dtype=np.float32)
        tot = C.c_double()
        L.check(self.num.lib.aslb_flux_compute(self.h, fld.ctypes.data_as(L._pf), C.byref(tot)),
                "ComputeSurfaceFlux::execute")
        return fld, tot.value

    def __del__(self):
        try:
            if self.h:
                self.num.lib.aslb_flux_destroy(self.h)
                self.h = None
        except Exception:
            pass


def generateComputeSurfaceFlux(lbgk: LBGK, m: np.ndarray) -> ComputeSurfaceFlux:
    return ComputeSurfaceFlux(lbgk, m)


class ComputeSurfaceForce:
    """ComputeSurfaceForceMap (src/num/aslLBGKBC.cxx:674-742) plus an FP64
    reduction to total force and torque about ``r0``."""

    def __init__(self, lbgk: LBGK, m: np.ndarray):
        self.num = lbgk
        arr = _map_array(lbgk, m)
        h = C.c_void_p()
        L.check(lbgk.lib.aslb_force_create(lbgk.h, arr.ctypes.data_as(L._pf), C.byref(h)), "ComputeSurfaceForce")
        self.h = h

    def init(self):
        pass

    def execute(self, r0=(0.0, 0.0, 0.0), field: bool = False):
        out = (C.c_double * 6)()
        fld = None
        if field:
            fld = np.zeros((3, *self.num.block.ghosted), dtype=np.float32)
        L.check(self.num.lib.aslb_force_compute(self.h, L.dvec(r0), None if fld is None else fld.ctypes.data_as(L._pf),
                                                out), "ComputeSurfaceForce::execute")
        res = np.array(out[:])
        return (res, fld) if field else res

    def __del__(self):
        try:
            if self.h:
                self.num.lib.aslb_force_destroy(self.h)
                self.h = None
        except Exception:
            pass


def generateComputeSurfaceForce(lbgk: LBGK, m: np.ndarray) -> ComputeSurfaceForce:
    return ComputeSurfaceForce(lbgk, m)


class Batch:
    """Extension (no ASL analogue): many independent LBGK domains advanced
    together, one stream-collide launch per step for all of them plus one link
    launch per condition position, replayed from a CUDA graph
    (aslb_batch_create / aslb_batch_run)."""

    def __init__(self, domains: Sequence[LBGK]):
        self.domains = list(domains)
        if not self.domains:
            raise L.ASLError("ASL ERROR: Batch: no domains")
        self.lib = self.domains[0].lib
        arr = (C.c_void_p * len(self.domains))(*[d.h.value if isinstance(d.h, C.c_void_p) else d.h
                                                  for d in self.domains])
        h = C.c_void_p()
        L.check(self.lib.aslb_batch_create(arr, len(self.domains), C.byref(h)), "Batch")
        self.h = h

    def run(self, nsteps: int, bcs: Sequence[Sequence["BC"]] = (), use_graph: bool = True):
        """`for n: for each domain: execute(); executeAll(its bcs)`, batched.
        ``bcs[i]``: the conditions of domain i, in ASL's order."""
        lists = list(bcs) if bcs else [[] for _ in self.domains]
        if len(lists) != len(self.domains):
            raise L.ASLError("ASL ERROR: Batch::run: one condition list per domain")
        flat = [b.h for lst in lists for b in lst]
        arr = (C.c_void_p * max(1, len(flat)))(*flat)
        counts = (C.c_int * len(lists))(*[len(lst) for lst in lists])
        L.check(self.lib.aslb_batch_run(self.h, int(nsteps), arr, counts, 1 if use_graph else 0), "Batch::run")

    def sync(self):
        L.check(self.lib.aslb_batch_sync(self.h), "Batch::sync")

    @property
    def tiles(self) -> int:
        return int(self.lib.aslb_batch_tiles(self.h))

    def setShape(self, shape: int):
        """Launch shape of the batched step (-1: chosen by timing, the default)."""
        L.check(self.lib.aslb_batch_set_shape(self.h, int(shape)), "Batch::setShape")

    @property
    def shape(self) -> int:
        return int(self.lib.aslb_batch_get_shape(self.h))

    @property
    def shape_times(self) -> list:
        buf = (C.c_float * 8)()
        n = int(self.lib.aslb_batch_shape_times(self.h, buf, 8))
        return [float(buf[i]) for i in range(min(n, 8))]

    def close(self):
        if getattr(self, "h", None):
            self.lib.aslb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def initAll(items):
    for it in items:
        it.init()


def executeAll(items):
    for it in items:
        it.execute()
