"""ctypes binding of ``include/pictor_b200.h``.

The library is the product: there is no CPU fallback.  Loading raises when
``libpictor_b200.so`` is absent, and every entry point raises ``PicError`` on
a nonzero return code.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

MAX_FLVR = 15

PIC_OK = 0
ERRORS = {
    -1: "PIC_ERR_INVALID", -2: "PIC_ERR_OOM", -3: "PIC_ERR_OVERFLOW", -4: "PIC_ERR_NAN",
    -5: "PIC_ERR_TIMEOUT", -6: "PIC_ERR_CUDA", -7: "PIC_ERR_RANGE", -8: "PIC_ERR_NOGPU",
}
PHASES = ("bhalf1", "move", "exchange", "bhalf2", "efield", "reorder")
GEOM = {"cartesian": 0, "cylindrical": 1}
FDTD = {"yee": 0, "lehe": 1}
PRECISION = {"fp64": 0, "fp32": 1}


class PicError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({_lib_error_string(code)})")


class Config(C.Structure):
    """pic_config: the runtime form of parameters.F90 + the species table."""

    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("dims", C.c_int32), ("geom", C.c_int32), ("fdtd", C.c_int32), ("precision", C.c_int32),
        ("nflvr", C.c_int32),
        ("c", C.c_double), ("qi", C.c_double), ("bext", C.c_double * 3),
        ("qm", C.c_double * (MAX_FLVR + 1)),
        ("reorder_period", C.c_int32), ("curr_filter", C.c_int32),
        ("capacity", C.c_int64),
        ("rmin", C.c_double), ("inc_axis", C.c_int32), ("brick", C.c_int32 * 3), ("cyl_modes", C.c_int32),
        ("slab_x", C.c_int32), ("exact_current", C.c_int32), ("fp64_tiles", C.c_int32),
        ("exact_charge", C.c_int32), ("reserved", C.c_int32 * 3),
    ]


class Inflow(C.Structure):
    """pic_inflow (include/pictor_b200.h)."""
    _fields_ = [
        ("face", C.c_int32), ("pos", C.c_double), ("speed", C.c_double), ("vmax", C.c_double),
        ("epc", C.c_double), ("density", C.c_double), ("drift", C.c_double * 3), ("nspecies", C.c_int32),
        ("flv", C.c_int32 * 4), ("temp", C.c_double * 4), ("charge", C.c_double * 4), ("seed", C.c_uint32),
        ("call", C.c_uint32),
    ]


_LIB = None


def library_path() -> str:
    return _build.LIB


def lib() -> C.CDLL:
    """Load libpictor_b200.so (built in-tree); raises if it is missing."""
    global _LIB
    if _LIB is None:
        path = library_path()
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: run pictor_b200.build.build() (nvcc) first")
        L = C.CDLL(path)
        _declare(L)
        _LIB = L
    return _LIB


def _lib_error_string(code: int) -> str:
    try:
        return lib().pic_error_string(code).decode()
    except Exception:  # the library itself may be what failed to load
        return "?"


PD = C.POINTER(C.c_double)
PI32 = C.POINTER(C.c_int32)
PI64 = C.POINTER(C.c_int64)
H = C.c_void_p

# name -> (restype, argtypes); every symbol declared in include/pictor_b200.h
SIGNATURES = {
    "pic_version": (C.c_int, []),
    "pic_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "pic_destroy": (None, [H]),
    "pic_load_fields": (C.c_int, [H] + [PD] * 6),
    "pic_fetch_fields": (C.c_int, [H] + [PD] * 9),
    "pic_load_current": (C.c_int, [H] + [PD] * 3),
    "pic_load_particles": (C.c_int, [H, C.c_int64] + [PD] * 7 + [PI32]),
    "pic_fetch_particles": (C.c_int, [H, PI64] + [PD] * 7 + [PI32]),
    "pic_particle_count": (C.c_int, [H, PI64]),
    "pic_init_weibel": (C.c_int, [H, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint32]),
    "pic_update_b_half": (C.c_int, [H]),
    "pic_move_deposit": (C.c_int, [H]),
    "pic_exchange_particles": (C.c_int, [H]),
    "pic_update_e": (C.c_int, [H]),
    "pic_fold_current": (C.c_int, [H]),
    "pic_add_current": (C.c_int, [H]),
    "pic_reset_current": (C.c_int, [H]),
    "pic_reorder": (C.c_int, [H]),
    "pic_filter_current": (C.c_int, [H]),
    "pic_slab_face_len": (C.c_int, [H, PI64]),
    "pic_set_sync": (C.c_int, [H, C.c_int32]),
    "pic_bc_reflect_x": (C.c_int, [H, C.c_int32, C.c_double]),
    "pic_bc_conducting_x": (C.c_int, [H, C.c_int32, C.c_double]),
    "pic_bc_reflect_y": (C.c_int, [H, C.c_int32, C.c_double]),
    "pic_bc_conducting_y": (C.c_int, [H, C.c_int32, C.c_double]),
    "pic_bc_remove": (C.c_int, [H, C.c_int32, C.c_double]),
    "pic_bc_attenuate": (C.c_int, [H, C.c_int32, PD, PD]),
    "pic_bc_attenuate_flow": (C.c_int, [H, C.c_int32, C.c_double, C.c_double, C.c_double, PD, PD]),
    "pic_bc_open_x": (C.c_int, [H, C.c_int32, C.c_double]),
    "pic_bc_open_prtl_x": (C.c_int, [H, C.c_int32, C.c_double]),
    "pic_solve_gauss": (C.c_int, [H, C.c_double, C.c_int32, C.POINTER(C.c_int32), PD, PD]),
    "pic_bc_inflow": (C.c_int, [H, C.POINTER(Inflow)]),
    "pic_bc_inflow_reflect": (C.c_int, [H, C.c_double, C.c_double]),
    "pic_bc_pml": (C.c_int, [H, C.c_int32, PD, PD]),
    "pic_slab_pack_particles_fixed": (C.c_int, [H, C.c_void_p, C.c_void_p, C.c_int64]),
    "pic_slab_unpack_particles_fixed": (C.c_int, [H, C.c_void_p, C.c_void_p, C.c_int64]),
    "pic_bc_pml_b": (C.c_int, [H]),
    "pic_bc_pml_e": (C.c_int, [H]),
    "pic_slab_pack_fields": (C.c_int, [H, C.c_int32, C.c_void_p, C.c_void_p]),
    "pic_slab_unpack_fields": (C.c_int, [H, C.c_int32, C.c_void_p, C.c_void_p]),
    "pic_slab_pack_particles": (C.c_int, [H, C.c_void_p, C.c_int64, PI64, PI64]),
    "pic_slab_unpack_particles": (C.c_int, [H, C.c_void_p, C.c_int64]),
    "pic_step": (C.c_int, [H, C.c_int32]),
    "pic_step_many": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32]),
    "pic_step_batched": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32]),
    "pic_step_persistent": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.c_uint32, C.c_int32]),
    "pic_set_step": (C.c_int, [H, C.c_int64]),
    "pic_diagnostics": (C.c_int, [H, C.c_double, PD, C.c_int32]),
    "pic_device_errors": (C.c_int, [H, PI32]),
    "pic_profile": (C.c_int, [H, C.c_int32]),
    "pic_phase_times": (C.c_int, [H, PD, PI64, C.c_int32, PI64]),
    "pic_launch_count": (C.c_int, [H, PI64]),
    "pic_field_energy_noalloc": (C.c_int, [C.c_void_p] * 6 + [C.c_int32] * 4 + [C.c_void_p, C.c_void_p]),
    "pic_adj_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "pic_adj_destroy": (None, [C.c_void_p]),
    "pic_adj_init_weibel": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_uint32, PI64]),
    "pic_adj_load_particles": (C.c_int, [C.c_void_p, C.c_int64] + [PD] * 7 + [PI32, PD]),
    "pic_adj_fetch_particles": (C.c_int, [C.c_void_p, PI64] + [PD] * 7 + [PI32, PD]),
    "pic_adj_forward": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, PD]),
    "pic_adj_branches": (C.c_int, [C.c_void_p, C.c_int32]),
    "pic_adj_gradient": (C.c_int, [C.c_void_p, C.c_double, PD, PD, PD, PD, PD, PD, PD]),
    "pic_error_string": (C.c_char_p, [C.c_int]),
    "pic_stream": (C.c_void_p, [H]),
}


def _declare(L: C.CDLL) -> None:
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def check(code: int, where: str) -> None:
    if code != PIC_OK:
        raise PicError(code, where)


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]), "float64 contiguous array required"
    return a.ctypes.data_as(PD)


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"], "int32 contiguous array required"
    return a.ctypes.data_as(PI32)
