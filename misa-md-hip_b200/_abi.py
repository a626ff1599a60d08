"""ctypes mirror of include/misa_b200.h.

Loads the in-tree ``libmisa_b200.so`` and declares every exported entry point.
There is no fallback: if the library is missing or fails to load, this module
raises, so no caller can silently run without the CUDA build.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "libmisa_b200.so"

MB_OK = 0
MB_ERR_ARG = 1
MB_ERR_CUDA = 2
MB_ERR_STATE = 3
MB_ERR_NOMEM = 4
MB_ERR_TIMEOUT = 5
MB_ERR_UNSUPPORTED = 6
MB_PREC_FP64 = 0
MB_PREC_MIXED = 1

# numpy view of mb_atom_element (104 bytes, the reference's _cuAtomElement)
ATOM_DTYPE = np.dtype([
    ("id", "<i8"), ("type", "<i4"), ("pad_", "<i4"),
    ("x", "<f8", (3,)), ("v", "<f8", (3,)), ("f", "<f8", (3,)),
    ("rho", "<f8"), ("df", "<f8"),
])
assert ATOM_DTYPE.itemsize == 104


class MbAtomElement(C.Structure):
    _fields_ = [("id", C.c_int64), ("type", C.c_int32), ("pad_", C.c_int32),
                ("x", C.c_double * 3), ("v", C.c_double * 3), ("f", C.c_double * 3),
                ("rho", C.c_double), ("df", C.c_double)]


class MbDeviceDomain(C.Structure):
    _fields_ = [("ghost_size_x", C.c_int32), ("ghost_size_y", C.c_int32), ("ghost_size_z", C.c_int32),
                ("box_size_x", C.c_int32), ("box_size_y", C.c_int32), ("box_size_z", C.c_int32),
                ("ext_size_x", C.c_int32), ("ext_size_y", C.c_int32), ("ext_size_z", C.c_int32),
                ("pad_", C.c_int32),
                ("box_index_start_x", C.c_int64), ("box_index_start_y", C.c_int64),
                ("box_index_start_z", C.c_int64)]


class MbEamTables(C.Structure):
    _fields_ = [("n_types", C.c_int32), ("nr", C.c_int32), ("nrho", C.c_int32), ("pad_", C.c_int32),
                ("dr", C.c_double), ("drho", C.c_double), ("cutoff", C.c_double),
                ("f", C.POINTER(C.c_double)), ("F", C.POINTER(C.c_double)), ("phi", C.POINTER(C.c_double))]


class MbSimConfig(C.Structure):
    _fields_ = [("cells_x", C.c_int32), ("cells_y", C.c_int32), ("cells_z", C.c_int32),
                ("precision", C.c_int32),
                ("lattice_const", C.c_double), ("mass", C.c_double), ("dt", C.c_double),
                ("cutoff", C.c_double), ("stencil_skin", C.c_double),
                ("max_interstitials", C.c_int32), ("pad_", C.c_int32)]


assert C.sizeof(MbAtomElement) == 104

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_PD = C.POINTER(C.c_double)
_PI64 = C.POINTER(C.c_int64)
_PI = C.POINTER(C.c_int)
_PF = C.POINTER(C.c_float)

# name -> (restype, argtypes); the exact set include/misa_b200.h declares
SIGNATURES: dict[str, tuple] = {
    "mb_last_error": (C.c_char_p, []),
    "mb_version": (C.c_char_p, []),
    "mb_env_init": (_I, [_I]),
    "mb_env_clean": (_I, []),
    "mb_domain_init": (_I, [C.POINTER(MbDeviceDomain)]),
    "mb_nei_offset_init": (_I, [_PI64, C.c_size_t, _PI64, C.c_size_t]),
    "mb_pot_init": (_I, [C.POINTER(MbEamTables)]),
    "mb_eam_rho_calc": (_I, [_P, _D]),
    "mb_eam_rho_calc_noalloc": (_I, [_P, _D]),
    "mb_eam_df_calc": (_I, [_P, _D]),
    "mb_eam_force_calc": (_I, [_P, _D]),
    "mb_eam_df_from_rho": (_I, [_P]),
    "mb_set_half_neighbour": (_I, [C.c_int]),
    "mb_create_atoms_mem": (_I, [C.POINTER(_P), C.c_size_t, C.c_int64, C.c_int64, C.c_int64, _PI]),
    "mb_release_atoms_mem": (_I, [_P, _PI]),
    "mb_cli_set_batches": (_I, [C.c_uint]),
    "mb_cli_batches": (C.c_uint, []),
    "mb_hook_last_timing": (_I, [_PF, _PF]),
    "mb_spline_coeffs": (_I, [_PD, _I, _D, _PD]),
    "mb_stencil_linear": (_I, [_D, _D, _I, _I, _PI64, _PI64, _I, _PI]),
    "mb_sim_create": (_I, [C.POINTER(MbSimConfig), C.POINTER(MbEamTables), C.POINTER(_P)]),
    "mb_sim_destroy": (_I, [_P]),
    "mb_sim_upload": (_I, [_P, _P, _P, C.c_int32]),
    "mb_sim_download": (_I, [_P, _P, _P, C.POINTER(C.c_int32)]),
    "mb_sim_run": (_I, [_P, C.c_int32, C.c_int32]),
    "mb_sim_sync": (_I, [_P]),
    "mb_sim_energies": (_I, [_P, _PD, C.c_int32, C.POINTER(C.c_int32)]),
    "mb_sim_time_steps": (_I, [_P, C.c_int32, _PF]),
    "mb_sim_step_host": (_I, [_P, _P, _P, C.c_int32]),
    "mb_sim_set_host_slabs": (_I, [_P, C.c_int32]),
    "mb_sim_host_slabs": (_I, [_P, C.POINTER(C.c_int32)]),
    "mb_sim_kernel_times": (_I, [_P, _PF, _PF]),
    "mb_sim_info": (_I, [_P, _PI64, _PI64, _PI64]),
    "mb_sim_set_graphs": (_I, [_P, _I]),
    "mb_sim_set_conversion": (_I, [_P, _D, _D]),
    "mb_sim_conversion_stats": (_I, [_P, _PI64, C.POINTER(C.c_int32)]),
    "mb_ensemble_set_conversion": (_I, [_P, _D, _D]),
    "mb_ensemble_conversion_stats": (_I, [_P, C.c_int32, _PI64, C.POINTER(C.c_int32)]),
    "mb_ensemble_create": (_I, [C.c_void_p, C.POINTER(MbEamTables), C.POINTER(_P)]),
    "mb_ensemble_destroy": (_I, [_P]),
    "mb_ensemble_lattice_bytes": (_I, [C.c_void_p, _PI64]),
    "mb_ensemble_add": (_I, [_P, C.c_void_p, _P, _P, C.c_int32, C.c_int64, C.POINTER(C.c_int32)]),
    "mb_ensemble_remove": (_I, [_P, C.c_int32]),
    "mb_ensemble_set_steps": (_I, [_P, C.c_int32, C.c_int64]),
    "mb_ensemble_advance": (_I, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "mb_ensemble_run": (_I, [_P, C.c_int32, C.c_int32]),
    "mb_ensemble_sync": (_I, [_P]),
    "mb_ensemble_download": (_I, [_P, C.c_int32, _P, _P, C.POINTER(C.c_int32)]),
    "mb_ensemble_status": (_I, [_P, C.c_int32, _PI64, _PI64, _PI64]),
    "mb_ensemble_energies": (_I, [_P, C.c_int32, _PD, C.c_int32, C.POINTER(C.c_int32)]),
    "mb_ensemble_clear_energies": (_I, [_P, C.c_int32]),
    "mb_ensemble_time": (_I, [_P, C.c_int32, _PF]),
    "mb_ensemble_set_policy": (_I, [_P, C.c_int32]),
    "mb_ensemble_autotune": (_I, [_P, C.c_int32, C.POINTER(C.c_int32), _PF]),
    "mb_ensemble_info": (_I, [_P, _PI64, _PI64, _PI64, C.POINTER(C.c_int32)]),
    "mb_ensemble_set_graphs": (_I, [_P, _I]),
    "mb_ensemble_set_wait_limit": (_I, [_P, C.c_int64]),
    "mb_sim_create_slab": (_I, [C.POINTER(MbSimConfig), C.POINTER(MbEamTables), C.c_int32, C.c_int32,
                                C.POINTER(_P)]),
    "mb_sim_halo_bytes": (_I, [_P, C.c_int32, _PI64]),
    "mb_sim_halo_pack": (_I, [_P, C.c_int32, C.c_int32, C.c_void_p]),
    "mb_sim_halo_unpack": (_I, [_P, C.c_int32, C.c_int32, C.c_void_p, _D]),
    "mb_sim_slab_phase": (_I, [_P, C.c_int32, C.c_int32]),
    "mb_sim_clear_energies": (_I, [_P]),
    "mb_ensemble_set_mode": (_I, [_P, C.c_int32]),
    "mb_ensemble_kernel_times": (_I, [_P, _PF, _PF, C.POINTER(C.c_int32)]),
}


class MbEnsembleConfig(C.Structure):
    _fields_ = [("lattice_const", C.c_double), ("mass", C.c_double), ("dt", C.c_double), ("cutoff", C.c_double),
                ("stencil_skin", C.c_double), ("hbm_budget_bytes", C.c_int64), ("max_lattices", C.c_int32),
                ("pad_", C.c_int32)]


class MbLatticeSpec(C.Structure):
    _fields_ = [("cells_x", C.c_int32), ("cells_y", C.c_int32), ("cells_z", C.c_int32),
                ("max_interstitials", C.c_int32)]

_lib = None


class MbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"misa_b200 error {code}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """The loaded library (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run misa-md-hip_b200/build.py (or __graft_entry__.build())")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != MB_OK:
        raise MbError(rc, lib().mb_last_error().decode())


def ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_PD)


def i64ptr(a: np.ndarray):
    assert a.dtype == np.int64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_PI64)
