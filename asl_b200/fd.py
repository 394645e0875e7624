"""FD advection-diffusion coupled to an LBGK velocity field (ASL's
FDAdvectionDiffusion, src/num/aslFDAdvectionDiffusion.cxx:88-180, 209-226).

``generateFDAdvectionDiffusion(c, D, v, vt, compressibilityCorrection)``
builds the solver on the GPU (``aslb_fd_*``): ``c`` is the ghosted initial
field (ASL layout, FP32 or FP64), ``v`` an LBGK whose velocity the solver
reads on the device (or None), ``vt`` the stencil template (d3q7, d3q15 or
d3q19). ``execute()`` advances one step on the LBGK's stream, after its
steps; ``generateBCConstantValue(fd, value, walls)`` fixes face ghost
layers (ghost values are never written by a step, as in ASL).
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Optional, Union

import numpy as np

from . import _lib as L
from .lbgk import LBGK, VectorTemplate


def _q(vt) -> int:
    q = vt.q if isinstance(vt, VectorTemplate) else int(vt)
    if q not in (7, 15, 19):
        raise L.ASLError("ASL ERROR: FDAdvectionDiffusion: template must be d3q7, d3q15 or d3q19")
    return q


class FDAdvectionDiffusion:
    def __init__(self, c: np.ndarray, D: float, vt: Union[VectorTemplate, int], velocity: Optional[LBGK] = None,
                 compressibilityCorrection: bool = False):
        self.lib = L.load()
        c = np.asarray(c)
        self.dtype = np.float64 if c.dtype == np.float64 else np.float32
        self.code = L.F64 if self.dtype == np.float64 else L.F32
        self.shape = c.shape
        nx, ny, nz = (s - 2 for s in c.shape)
        h = C.c_void_p()
        L.check(self.lib.aslb_fd_create(nx, ny, nz, _q(vt), self.code, float(D), C.byref(h)), "FDAdvectionDiffusion")
        self.h = h
        self.velocity = velocity
        self._c0 = np.ascontiguousarray(c, dtype=self.dtype)
        if velocity is not None:
            L.check(self.lib.aslb_fd_set_velocity(self.h, velocity.h, int(bool(compressibilityCorrection))),
                    "FDAdvectionDiffusion::setVelocity")
        self.setC(self._c0)

    def init(self):
        pass

    def setC(self, c: np.ndarray):
        c = np.ascontiguousarray(c, dtype=self.dtype)
        if c.shape != self.shape:
            raise L.ASLError("ASL ERROR: FDAdvectionDiffusion: field of another shape")
        L.check(self.lib.aslb_fd_write(self.h, self.code, c.ctypes.data_as(C.c_void_p)), "FDAdvectionDiffusion")

    def getC(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=self.dtype)
        L.check(self.lib.aslb_fd_read(self.h, self.code, out.ctypes.data_as(C.c_void_p)), "FDAdvectionDiffusion")
        return out

    def setElectricFieldParameters(self, phi: np.ndarray, k: np.ndarray, f2=None, q: np.ndarray = None):
        """c' -= divAgradB(c q / k, phi) each step (ASL's f2 is unused there)."""
        arrs = [np.ascontiguousarray(a, dtype=self.dtype) for a in (phi, k, q)]
        if any(a.shape != self.shape for a in arrs):
            raise L.ASLError("ASL ERROR: setElectricFieldParameters: fields of another shape")
        self._ef = arrs
        L.check(self.lib.aslb_fd_set_electric_field(self.h, self.code, *[a.ctypes.data_as(C.c_void_p) for a in arrs]),
                "FDAdvectionDiffusion::setElectricFieldParameters")

    def setDiffusionCoefficient(self, D: float):
        L.check(self.lib.aslb_fd_set_diffusion(self.h, float(D)), "FDAdvectionDiffusion")

    def execute(self, n: int = 1):
        L.check(self.lib.aslb_fd_step(self.h, int(n)), "FDAdvectionDiffusion::execute")

    def sync(self):
        L.check(self.lib.aslb_fd_sync(self.h), "FDAdvectionDiffusion")

    def close(self):
        if getattr(self, "h", None):
            self.lib.aslb_fd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generateFDAdvectionDiffusion(c, D: float, v=None, vt=7, compressibilityCorrection: bool = False):
    return FDAdvectionDiffusion(c, D, vt, v, compressibilityCorrection)


class FDMapBC:
    """A condition on the FD field at a map surface; ``execute()`` after each
    FD step, as ASL's executeAll(bc)."""

    def __init__(self, fd: FDAdvectionDiffusion, kind: int, m: np.ndarray, value: float):
        m = np.ascontiguousarray(m, dtype=np.float32)
        if m.shape != fd.shape:
            raise L.ASLError("ASL ERROR: map must cover the FD field's ghosted block")
        self.fd = fd
        h = C.c_void_p()
        L.check(fd.lib.aslb_fd_bc_create(fd.h, kind, m.ctypes.data_as(C.c_void_p), float(value), C.byref(h)),
                "generateBC")
        self.h = h

    def init(self):
        pass

    def execute(self):
        L.check(self.fd.lib.aslb_fd_bc_execute(self.h), "BC::execute")

    @property
    def cells(self) -> int:
        return int(self.fd.lib.aslb_fd_bc_cells(self.h))

    def __del__(self):
        try:
            if self.h:
                self.fd.lib.aslb_fd_bc_destroy(self.h)
                self.h = None
        except Exception:
            pass


def generateBCConstantValue(fd: FDAdvectionDiffusion, value: float, where):
    """BCConstantValue on faces (src/num/aslBasicBC.cxx:51-57): the ghost
    layers of the given faces hold ``value`` (applied at once, never
    overwritten by a step); on a map (BCConstantValueMap, :71-108) a
    condition object whose ``execute()`` sets the guard cells to ``value``."""
    if isinstance(where, np.ndarray):
        return FDMapBC(fd, 0, where, value)
    mask = 0
    for w in where:
        mask |= 1 << int(w)
    L.check(fd.lib.aslb_fd_set_face_value(fd.h, mask, float(value)), "generateBCConstantValue")


def generateBCConstantGradient(fd: FDAdvectionDiffusion, value: float, m: np.ndarray) -> FDMapBC:
    """BCConstantGradientMap (src/num/aslBasicBC.cxx:271-350) on the FD's
    template: the guard cells take the normal gradient ``value``."""
    return FDMapBC(fd, 1, m, value)
