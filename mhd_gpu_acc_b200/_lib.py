"""ctypes binding of libmhd_b200.so (the C ABI declared in include/mhd_b200.h).

The library is built in-tree (``python -m mhd_gpu_acc_b200.build``).  There is
no Python fallback: if the shared library is missing, loading fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmhd_b200.so")

MHD_OK = 0
ERRORS = {
    -1: "MHD_ERR_ARG",
    -2: "MHD_ERR_CUDA",
    -3: "MHD_ERR_NO_SPEED",
    -4: "MHD_ERR_BAD_DT",
    -5: "MHD_ERR_TINY_DT",
    -6: "MHD_ERR_STATE",
    -7: "MHD_ERR_NOMEM",
    -8: "MHD_ERR_TIMEOUT",
}


class mhd_grid(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("pitch", C.c_longlong),
        ("plane", C.c_longlong),
        ("nx", C.c_int),
        ("ny", C.c_int),
        ("ng", C.c_int),
        ("dtype", C.c_int),
        ("x_min", C.c_double),
        ("x_max", C.c_double),
        ("y_min", C.c_double),
        ("y_max", C.c_double),
    ]


class mhd_run_info(C.Structure):
    _fields_ = [
        ("t", C.c_double),
        ("last_dt", C.c_double),
        ("ch", C.c_double),
        ("steps", C.c_int),
        ("status", C.c_int),
        ("fallbacks", C.c_uint),
        ("pad_", C.c_uint),
    ]


class mhd_state_meta(C.Structure):
    _fields_ = [("t", C.c_double), ("ch", C.c_double), ("steps", C.c_longlong)]


class mhd_instance_desc(C.Structure):
    _fields_ = [
        ("nx", C.c_int),
        ("ny", C.c_int),
        ("ng", C.c_int),
        ("bc", C.c_int * 4),
        ("x_min", C.c_double),
        ("x_max", C.c_double),
        ("y_min", C.c_double),
        ("y_max", C.c_double),
        ("gamma", C.c_double),
        ("cfl", C.c_double),
        ("cr", C.c_double),
        ("t_end", C.c_double),
    ]


class mhd_batch_tuning(C.Structure):
    _fields_ = [("xrpw", C.c_int), ("yseg", C.c_int), ("ctas_x", C.c_int), ("ctas_y", C.c_int)]


_D, _I, _P = C.c_double, C.c_int, C.c_void_p
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)
_pg = C.POINTER(mhd_grid)

# name -> (restype, argtypes); every entry point of include/mhd_b200.h
PROTOTYPES = {
    "mhd_grid_alloc": (_I, [_pg, _I, _I, _I, _I, _D, _D, _D, _D]),
    "mhd_grid_free": (_I, [_pg]),
    "mhd_grid_upload": (_I, [_pg, _P]),
    "mhd_grid_download": (_I, [_pg, _P]),
    "mhd_grid_upload_aos": (_I, [_pg, _P]),
    "mhd_grid_download_aos": (_I, [_pg, _P]),
    "mhd_grid_swap": (_I, [_pg, _pg]),
    "mhd_workspace_create": (_I, [_pg, C.POINTER(_P)]),
    "mhd_workspace_destroy": (_I, [_P]),
    "mhd_workspace_set_stream": (_I, [_P, _P]),
    "mhd_set_gamma": (_I, [_P, _D]),
    "mhd_set_ch": (_I, [_P, _D]),
    "mhd_get_ch": (_I, [_P, _pd]),
    "mhd_set_limiter": (_I, [_P, _I]),
    "mhd_set_cr": (_I, [_P, _D]),
    "mhd_set_sweep_shape": (_I, [_P, _I, _I, _I]),
    "mhd_set_tma_wait_limit": (_I, [_P, C.c_ulonglong]),
    "mhd_set_spacing": (_I, [_P, _D, _D]),
    "mhd_compute_dt": (_I, [_P, _pg, _D, _pd]),
    "mhd_advance": (_I, [_P, _pg, _pg, _pg, _D, _I, _pi]),
    "mhd_apply_boundary": (_I, [_P, _pg, _pi]),
    "mhd_sweep": (_I, [_P, _pg, _pg, _D, _I, _pi, _I]),
    "mhd_max_speed": (_I, [_P, _pg, _pd]),
    "mhd_grid_copy_rows": (_I, [_pg, _I, _pg, _I, _I, _P]),
    "mhd_advance_noalloc": (_I, [_pg, _pg, _D, _D, _D, _D, _I, _I, _pi, _P]),
    "mhd_clock_start": (_I, [_P, _pg, _D, _D]),
    "mhd_clock_slot": (_I, [_P, _I, C.POINTER(_P)]),
    "mhd_sweep_clocked": (_I, [_P, _pg, _pg, _I, _pi, _I, _I, _I, _I, _I]),
    "mhd_clock_read": (_I, [_P, C.POINTER(mhd_run_info)]),
    "mhd_state_save": (_I, [_pg, C.c_char_p, C.POINTER(mhd_state_meta)]),
    "mhd_state_load": (_I, [_pg, C.c_char_p, C.POINTER(mhd_state_meta)]),
    "mhd_run": (_I, [_P, _pg, _pg, _D, _D, _I, _I, _pi, C.POINTER(mhd_run_info)]),
    "mhd_profile_sweeps": (_I, [_P, _pg, _pg, _D, _D, _I, _pi, _I, C.POINTER(C.c_float)]),
    "mhd_upload": (_I, [_P, _pg, _P]),
    "mhd_download": (_I, [_P, _pg, _P]),
    "mhd_upload_f32": (_I, [_P, _pg, _P]),
    "mhd_download_f32": (_I, [_P, _pg, _P]),
    "mhd_synchronize": (_I, [_P]),
    "mhd_diagnostics": (_I, [_P, _pg, _pd]),
    "mhd_case_config": (_I, [_I, _I, _pd]),
    "mhd_initial_state": (_I, [_I, _D, _D, _pd]),
    "mhd_initialise": (_I, [_I, _I, _I, _I, _D, _D, _D, _D, _P]),
    "mhd_riemann_flux": (_I, [_P, _P, _I, _I, _D, _D, _P]),
    "mhd_riemann_flux_device": (_I, [_P, _I, C.c_longlong, _P, _P, _I, _I, _D, _D, _P]),
    "mhd_initialise_device": (_I, [_P, _pg, _I]),
    "mhd_initialise_orszag_tang": (_I, [_P, _pg, _D, _D, _P]),
    "mhd_batch_create": (_I, [C.POINTER(mhd_instance_desc), _I, _I, _I, _I, C.POINTER(_P)]),
    "mhd_batch_destroy": (_I, [_P]),
    "mhd_batch_set_stream": (_I, [_P, _P]),
    "mhd_batch_grid": (_I, [_P, _I, _pg]),
    "mhd_batch_cells": (_I, [_P, C.POINTER(C.c_longlong)]),
    "mhd_batch_run": (_I, [_P, _I, C.POINTER(mhd_run_info)]),
    "mhd_batch_get_tuning": (_I, [_P, C.POINTER(mhd_batch_tuning)]),
    "mhd_batch_set_tuning": (_I, [_P, C.POINTER(mhd_batch_tuning)]),
    "mhd_batch_tune": (_I, [_P, _I, C.POINTER(mhd_batch_tuning)]),
    "mhd_batch_tune_candidates": (_I, [_I, _pi, _I]),
    "mhd_adjoint_create": (_I, [_I, _I, _I, _I, _D, _D, _D, _I, _I, C.POINTER(_P)]),
    "mhd_adjoint_destroy": (_I, [_P]),
    "mhd_adjoint_set_solver": (_I, [_P, _I]),
    "mhd_adjoint_set_target": (_I, [_P, _P]),
    "mhd_adjoint_forward": (_I, [_P, _P, _pd, _P]),
    "mhd_adjoint_gradient": (_I, [_P, _P, _pd, _P]),
    "mhd_last_error": (C.c_char_p, []),
    "mhd_version": (C.c_char_p, []),
    "mhd_launch_count": (C.c_ulonglong, []),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the library once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m mhd_gpu_acc_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MhdError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)}: {msg}")
        self.code = code


def check(code: int, where: str) -> int:
    if code != MHD_OK:
        raise MhdError(code, where, (load().mhd_last_error() or b"").decode())
    return code
