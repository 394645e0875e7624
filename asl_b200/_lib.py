"""ctypes binding of libaslb.so (the C ABI declared in include/aslb.h).

The shared library is built in-tree by ``asl_b200.build``. Importing this
module on a machine without the built library raises immediately: there is no
CPU fallback for the compute path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libaslb.so"

ASLB_OK = 0
F32, F16, F64 = 0, 1, 2
NO_VELOCITY, NO_RHO, INCOMPRESSIBLE = 1, 2, 4
PERIODIC_X, PERIODIC_Y, PERIODIC_Z = 8, 16, 32
PACKED_ROWS = 64
CLOSURE_NONE, CLOSURE_ASL_INTENT, CLOSURE_SMAGORINSKY, CLOSURE_MLP = 0, 1, 2, 3
BC_NOSLIP, BC_VELOCITY, BC_PRESSURE, BC_PRESSURE_VELOCITY = 0, 1, 2, 3
BC_MAP_NOSLIP, BC_MAP_VELOCITY, BC_MAP_VELOCITY_ROTATION, BC_MAP_PRESSURE_VELOCITY = 10, 11, 12, 13
BC_MAP_TRANSPORT_DEPOSITION, BC_MAP_KINETICS_DEPOSITION = 14, 15
BC_FIELD_NOSLIP_VEL, BC_FIELD_NOSLIP_RHO, BC_FIELD_VELOCITY_VEL, BC_FIELD_VELOCITY_VEL_ROTATION = 20, 21, 22, 23
FIELD_RHO, FIELD_VELOCITY, FIELD_F, FIELD_CS2 = 0, 1, 2, 3


class ASLError(RuntimeError):
    """Raised on a non-zero status, with ASL's error-message prefix
    (src/aslUtilities.cxx:68-95 of the reference throws "ASL ERROR: ...")."""


_vp = C.c_void_p
_pd = C.POINTER(C.c_double)
_pf = C.POINTER(C.c_float)

# name: (restype, argtypes)
PROTOTYPES = {
    "aslb_last_error": (C.c_char_p, []),
    "aslb_version": (C.c_char_p, []),
    "aslb_set_device": (C.c_int, [C.c_int]),
    "aslb_synchronize": (C.c_int, []),
    "aslb_lbgk_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint,
                                   C.POINTER(_vp)]),
    "aslb_lbgk_destroy": (C.c_int, [_vp]),
    "aslb_lbgk_stream": (_vp, [_vp]),
    "aslb_lbgk_set_stream": (C.c_int, [_vp, _vp]),
    "aslb_lbgk_set_viscosity": (C.c_int, [_vp, C.c_double]),
    "aslb_lbgk_get_viscosity": (C.c_double, [_vp]),
    "aslb_lbgk_set_compressible": (C.c_int, [_vp, C.c_int]),
    "aslb_lbgk_set_omega": (C.c_int, [_vp, _pd]),
    "aslb_lbgk_set_macro_output": (C.c_int, [_vp, C.c_int, C.c_int]),
    "aslb_lbgk_request_macro": (C.c_int, [_vp]),
    "aslb_lbgk_set_body_force": (C.c_int, [_vp, _pd]),
    "aslb_lbgk_set_closure": (C.c_int, [_vp, C.c_int, C.c_double]),
    "aslb_mlp_layout_bytes": (C.c_size_t, []),
    "aslb_lbgk_set_mlp": (C.c_int, [_vp, _vp, C.c_size_t]),
    "aslb_lbgk_set_fp16_scale": (C.c_int, [_vp, C.c_double]),
    "aslb_lbgk_set_position": (C.c_int, [_vp, _pd, C.c_double]),
    "aslb_lbgk_shape": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "aslb_lbgk_init_f": (C.c_int, [_vp, C.c_double, _pd]),
    "aslb_lbgk_init_f_fields": (C.c_int, [_vp, _pd, _pd]),
    "aslb_lbgk_compute_macro": (C.c_int, [_vp, C.c_int, C.c_int]),
    "aslb_lbgk_bind_velocity": (C.c_int, [_vp, _vp]),
    "aslb_lbgk_step_planes": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "aslb_lbgk_step_commit": (C.c_int, [_vp]),
    "aslb_lbgk_step": (C.c_int, [_vp, C.c_int]),
    "aslb_lbgk_run": (C.c_int, [_vp, C.c_int, C.POINTER(_vp), C.c_int, C.c_int]),
    "aslb_lbgk_sync": (C.c_int, [_vp]),
    "aslb_lbgk_set_kernel": (C.c_int, [_vp, C.c_int]),
    "aslb_lbgk_get_kernel": (C.c_int, [_vp]),
    "aslb_lbgk_steps": (C.c_longlong, [_vp]),
    "aslb_lbgk_read": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "aslb_lbgk_write": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "aslb_bc_map_create_cd": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_double, _pd, _pd, _pd, _vp]),
    "aslb_lbgk_watchdog": (C.c_int, [_vp, _pd]),
    "aslb_lattice": (C.c_int, [C.c_int, _vp, _vp, _vp]),
    "aslb_bc_field_create": (C.c_int, [_vp, C.c_int, _vp, _pd, _pd, _pd, _vp]),
    "aslb_bc_deposition_create": (C.c_int, [_vp, C.c_int, _vp, C.c_double, C.c_double, C.c_double, _vp]),
    "aslb_flux_create": (C.c_int, [_vp, _vp, _vp]),
    "aslb_flux_compute": (C.c_int, [_vp, _vp, _vp]),
    "aslb_flux_destroy": (C.c_int, [_vp]),
    "aslb_fd_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _vp]),
    "aslb_fd_set_velocity": (C.c_int, [_vp, _vp, C.c_int]),
    "aslb_fd_set_diffusion": (C.c_int, [_vp, C.c_double]),
    "aslb_fd_set_electric_field": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp]),
    "aslb_fd_write": (C.c_int, [_vp, C.c_int, _vp]),
    "aslb_fd_read": (C.c_int, [_vp, C.c_int, _vp]),
    "aslb_fd_set_face_value": (C.c_int, [_vp, C.c_uint, C.c_double]),
    "aslb_fd_bc_create": (C.c_int, [_vp, C.c_int, _vp, C.c_double, _vp]),
    "aslb_fd_bc_execute": (C.c_int, [_vp]),
    "aslb_fd_bc_cells": (C.c_longlong, [_vp]),
    "aslb_fd_bc_destroy": (C.c_int, [_vp]),
    "aslb_fd_step": (C.c_int, [_vp, C.c_int]),
    "aslb_fd_sync": (C.c_int, [_vp]),
    "aslb_fd_device_field": (_vp, [_vp]),
    "aslb_fd_destroy": (C.c_int, [_vp]),
    "aslb_read_stl": (C.c_int, [C.c_char_p, _vp, C.c_longlong, _vp]),
    "aslb_surface_map": (C.c_int, [_vp, C.c_longlong, C.c_int, C.c_int, C.c_int, _pd, C.c_double, C.c_double,
                                   C.c_int, C.c_double, C.c_double, _vp]),
    "aslb_lbgk_state_bytes": (C.c_size_t, [_vp]),
    "aslb_lbgk_save_state": (C.c_int, [_vp, _vp, C.c_size_t, _vp]),
    "aslb_lbgk_load_state": (C.c_int, [_vp, _vp, C.c_size_t, _vp]),
    "aslb_lbgk_device_field": (_vp, [_vp, C.c_int]),
    "aslb_lbgk_moments": (C.c_int, [_vp, _pd]),
    "aslb_bc_slice_create": (C.c_int, [_vp, C.c_int, C.c_uint, C.c_double, _pd, C.POINTER(_vp)]),
    "aslb_bc_map_create": (C.c_int, [_vp, C.c_int, _pf, C.c_double, _pd, _pd, _pd, C.POINTER(_vp)]),
    "aslb_bc_fuse": (C.c_int, [_vp]),
    "aslb_bc_is_fused": (C.c_int, [_vp]),
    "aslb_bc_execute": (C.c_int, [_vp]),
    "aslb_bc_destroy": (C.c_int, [_vp]),
    "aslb_bc_num_links": (C.c_longlong, [_vp]),
    "aslb_bc_kernels": (C.c_int, [_vp]),
    "aslb_force_create": (C.c_int, [_vp, _pf, C.POINTER(_vp)]),
    "aslb_force_compute": (C.c_int, [_vp, _pd, _pf, _pd]),
    "aslb_force_destroy": (C.c_int, [_vp]),
    "aslb_force_compute_noalloc": (C.c_int, [_vp, _pd, _pd]),
    "aslb_lbgk_set_mlp_period": (C.c_int, [_vp, C.c_int]),
    "aslb_lbgk_closure_features": (C.c_int, [_vp, _vp]),
    "aslb_mlp_param_count": (C.c_int, []),
    "aslb_mlp_grad_scratch_floats": (C.c_size_t, []),
    "aslb_mlp_grad": (C.c_int, [_vp, _vp, _vp, C.c_longlong, _vp, C.c_float, _vp, _vp, _vp]),
    "aslb_mlp_adam": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, _vp]),
    "aslb_mlp_pack": (C.c_int, [_vp, _vp, C.c_float, _vp]),
    "aslb_lbgk_halo_bytes": (C.c_size_t, [_vp]),
    "aslb_lbgk_halo_pack": (C.c_int, [_vp, C.c_int, _vp]),
    "aslb_lbgk_halo_unpack": (C.c_int, [_vp, C.c_int, _vp]),
    "aslb_lbgk_parity": (C.c_int, [_vp]),
    "aslb_batch_create": (C.c_int, [C.POINTER(_vp), C.c_int, C.POINTER(_vp)]),
    "aslb_batch_run": (C.c_int, [_vp, C.c_int, C.POINTER(_vp), C.POINTER(C.c_int), C.c_int]),
    "aslb_batch_sync": (C.c_int, [_vp]),
    "aslb_batch_tiles": (C.c_longlong, [_vp]),
    "aslb_batch_destroy": (C.c_int, [_vp]),
    "aslb_batch_set_shape": (C.c_int, [_vp, C.c_int]),
    "aslb_batch_get_shape": (C.c_int, [_vp]),
    "aslb_batch_shape_times": (C.c_int, [_vp, C.POINTER(C.c_float), C.c_int]),
    "aslb_geom_pack_spheres": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_ulonglong, C.c_int, C.c_int, C.c_int, _pd, _pd, C.POINTER(C.c_int)]),
}

_lib = None


def load() -> C.CDLL:
    """Load libaslb.so once and declare every prototype; raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ASLError(f"ASL ERROR: {LIB_PATH} is not built (python -m asl_b200.build); "
                       "the LBGK path has no CPU fallback")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str = "") -> None:
    if rc != ASLB_OK:
        msg = load().aslb_last_error().decode(errors="replace")
        raise ASLError(f"ASL ERROR: {what}: {msg} (status {rc})" if what else f"ASL ERROR: {msg} (status {rc})")


def dvec(v) -> C.Array:
    v = list(v)
    return (C.c_double * len(v))(*[float(a) for a in v])
