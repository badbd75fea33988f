"""ctypes binding of libawcm_b200.so (the C-ABI declared in include/awcm_b200.h).

There is no CPU fallback: if the library or a CUDA device is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libawcm_b200.so")

AWCM_OK = 0
STATUS_NAMES = {1: "ERR_ARG", 2: "ERR_OOM", 3: "ERR_CUDA", 4: "ERR_TIMEOUT", 5: "ERR_NONFINITE", 6: "ERR_STATE"}

c_int, c_double, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
P_double = ctypes.POINTER(ctypes.c_double)
P_int = ctypes.POINTER(ctypes.c_int)
P_u8 = ctypes.POINTER(ctypes.c_uint8)

# name -> argtypes (every entry point returns int status unless listed in _RESTYPES)
_SIGS = {
    "awcm2d_create": [c_int, c_int, c_int, c_double, c_double, c_double, c_double, c_int, ctypes.POINTER(c_void_p)],
    "awcm2d_destroy": [c_void_p],
    "awcm2d_dims": [c_void_p, P_int, P_int],
    "awcm2d_set_q": [c_void_p, P_double],
    "awcm2d_get_q": [c_void_p, P_double],
    "awcm2d_get_masks": [c_void_p, P_u8],
    "awcm2d_set_masks": [c_void_p, P_u8],
    "awcm2d_get_levels": [c_void_p, P_int],
    "awcm2d_set_levels": [c_void_p, P_int],
    "awcm2d_init_problem": [c_void_p, c_int, c_double, c_double],
    "awcm2d_prepare": [c_void_p, c_double],
    "awcm2d_fwt": [c_void_p, c_double],
    "awcm2d_iwt": [c_void_p, c_int],
    "awcm2d_interpolate": [c_void_p, c_int, c_int],
    "awcm2d_interpolate_all": [c_void_p, c_int],
    "awcm2d_create_scalar": [c_int, c_int, c_int, c_double, c_double, c_double, c_double, ctypes.POINTER(c_void_p)],
    "awcm2d_scalar_set_q": [c_void_p, P_double],
    "awcm2d_scalar_get_q": [c_void_p, P_double],
    "awcm2d_scalar_advance": [c_void_p, c_double, c_double, c_double, c_int, P_double],
    "awcm2d_manager": [c_void_p, c_int, c_int, c_int],
    "awcm2d_apply_bc": [c_void_p, c_double],
    "awcm2d_step": [c_void_p, c_double, c_double, c_double, c_double, c_double, P_double],
    "awcm2d_advance": [c_void_p, c_double, c_double, c_double, c_double, c_int, P_double],
    "awcm2d_launches_per_step": [c_void_p, P_int],
    "awcm2d_step_io_bytes": [c_void_p, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)],
    "awcm2d_stream": [c_void_p, ctypes.POINTER(c_void_p)],
    "awcm2d_set_prepare_mode": [c_void_p, c_int],
    "awcm2d_set_spin_limit": [c_void_p, ctypes.c_uint],
    "awcm2d_profile_step": [c_void_p, c_double, c_double, c_double, c_double, P_double],
    "awcm_measure_fp64_peak": [c_int, c_int, P_double],
    "awcm2d_profile_kernels": [c_void_p, c_double, c_double, c_double, c_double, c_int, ctypes.c_char_p, P_double, P_int],
    "awcm2d_frozen_run": [c_void_p, c_double, c_double, c_int, c_int, P_double],
    "awcm2d_adjoint": [c_void_p, c_double, c_double, c_int, c_int, c_int, P_double, P_double, P_double],
    "awcm2d_set_wenoz": [c_void_p, c_double, c_double],
    "awcm2d_get_geometry": [c_void_p, c_void_p],
    "awcm2d_save_state": [c_void_p, ctypes.c_char_p, c_double, ctypes.c_longlong],
    "awcm2d_load_state": [c_void_p, ctypes.c_char_p, P_double, ctypes.POINTER(ctypes.c_longlong)],
    "awcm2d_get_alpha_tape": [c_void_p, c_int, P_double],
    "awcm2d_set_alpha_tape": [c_void_p, c_int, P_double],
    "awcm1d_batch_create": [c_int, P_int, P_int, P_double, P_double, c_double, c_int, ctypes.POINTER(c_void_p)],
    "awcm1d_batch_destroy": [c_void_p],
    "awcm1d_batch_count": [c_void_p, P_int],
    "awcm1d_batch_nx": [c_void_p, c_int, P_int],
    "awcm1d_batch_set_q": [c_void_p, c_int, P_double],
    "awcm1d_batch_get_q": [c_void_p, c_int, P_double],
    "awcm1d_batch_get_masks": [c_void_p, c_int, P_u8],
    "awcm1d_batch_set_masks": [c_void_p, c_int, P_u8],
    "awcm1d_batch_get_levels": [c_void_p, c_int, P_int],
    "awcm1d_batch_set_levels": [c_void_p, c_int, P_int],
    "awcm1d_batch_init_riemann": [c_void_p, c_int, c_double, P_double, P_double],
    "awcm1d_batch_set_run": [c_void_p, P_double, P_double, P_double, P_double, c_double],
    "awcm1d_batch_steps": [c_void_p, c_int],
    "awcm1d_batch_run": [c_void_p, c_int],
    "awcm1d_batch_sync": [c_void_p],
    "awcm1d_batch_status": [c_void_p, c_int, P_double],
    "awcm1d_batch_totals": [c_void_p, P_double],
    "awcm1d_batch_pass": [c_void_p, c_int, c_int, c_int, c_int],
    "awcm1d_batch_prepare": [c_void_p, c_int, c_double],
    "awcm1d_batch_fwt": [c_void_p, c_int, c_double],
    "awcm1d_batch_iwt": [c_void_p, c_int, c_int],
    "awcm1d_batch_interpolate": [c_void_p, c_int, c_int, c_int],
    "awcm1d_batch_manager": [c_void_p, c_int, c_int, c_int, c_int],
    "awcm1d_batch_apply_bc": [c_void_p, c_int],
    "awcm1d_batch_set_bc_field": [c_void_p, c_int, P_int],
    "awcm2d_set_bc_field": [c_void_p, P_int],
    "awcm2d_wt_set_bottom": [c_void_p, c_int, c_int],
    "awcm1d_batch_set_launch": [c_void_p, c_int, c_int],
    "awcm1d_batch_stream": [c_void_p, ctypes.POINTER(c_void_p)],
    "awcm1d_step_noalloc": [c_int, c_int, c_double, c_double, c_double, c_int, c_double, c_double, c_double, c_double,
                            c_void_p, c_void_p, c_void_p, c_void_p],
    "euler1d_flux": [c_void_p, c_void_p, c_int, c_double, c_void_p],
    "euler1d_spectral_radius": [c_void_p, c_void_p, c_int, c_double, c_void_p],
    "euler2d_flux": [c_void_p, c_void_p, c_int, c_int, c_double, c_void_p],
    "euler2d_spectral_radius": [c_void_p, c_void_p, c_int, c_int, c_double, c_void_p],
    "awcm_last_error": [],
    "awcm_version": [],
}
_RESTYPES = {"awcm_last_error": ctypes.c_char_p, "awcm_version": ctypes.c_char_p}


class AwcmError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, name: str, status: int, message: str):
        super().__init__(f"{name} -> {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def exported_symbols() -> list[str]:
    return [n for n in _SIGS]


def load() -> ctypes.CDLL:
    """Loads the CUDA library (built by c_pp-library_b200/build.py); raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA extension missing: {LIB_PATH} (run python c_pp-library_b200/build.py)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = _RESTYPES.get(name, c_int)
        _lib = lib
    return _lib


def call(name: str, *args) -> None:
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != AWCM_OK:
        msg = lib.awcm_last_error().decode(errors="replace")
        raise AwcmError(name, rc, msg)


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))
