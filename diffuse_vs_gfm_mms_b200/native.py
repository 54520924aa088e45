"""Loader of the in-tree CUDA library libdimgpu.so (built by build.py).

There is no CPU fallback: importing the solver without the library, or
calling it on a machine without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libdimgpu.so")

# name -> (argtypes, restype)
_D = C.POINTER(abi.Desc)
_S = C.c_void_p
_DP = abi.DPTR
SIGNATURES = {
    "dimgpu_components": ([_D], C.c_int),
    "dimgpu_create": ([_D, C.POINTER(C.c_void_p)], C.c_int),
    "dimgpu_destroy": ([_S], C.c_int),
    "dimgpu_last_error": ([_S], C.c_char_p),
    "dimgpu_upload": ([_S, _DP, C.c_size_t], C.c_int),
    "dimgpu_download": ([_S, _DP, C.c_size_t], C.c_int),
    "dimgpu_step": ([_S, C.c_double, C.c_double, _DP, C.POINTER(abi.PhaseTimes)], C.c_int),
    "dimgpu_steps": ([_S, C.c_int, C.c_double, C.c_double, _DP], C.c_int),
    "dimgpu_enqueue_steps": ([_S, C.c_int, C.c_double, C.c_double], C.c_int),
    "dimgpu_collect": ([_S, _DP, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "dimgpu_compute_dt_cfl": ([_S, C.c_double, C.c_double, _DP], C.c_int),
    "dimgpu_sweep_direction": ([_S, C.c_int, C.c_double], C.c_int),
    "dimgpu_apply_boundary_conditions": ([_S], C.c_int),
    "dimgpu_totals": ([_S, _DP], C.c_int),
    "dimgpu_boundary_flux": ([_S, _DP], C.c_int),
    "dimgpu_set_stream": ([_S, C.c_void_p], C.c_int),
    "dimgpu_set_tile": ([_S, C.c_int, C.c_int, C.c_int], C.c_int),
    "dimgpu_set_schedule": ([_S, C.c_int, C.c_int], C.c_int),
    "dimgpu_profile": ([_S, C.c_int], C.c_int),
    "dimgpu_profile_read": ([_S, _DP], C.c_int),
    "dimgpu_kernel_launches": ([], C.c_longlong),
    "dimgpu_compute_dt_cfl_noalloc": ([_D, _DP, C.c_double, C.c_double, _DP, C.c_void_p], C.c_int),
    "dimgpu_batch_create": ([C.c_int, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "dimgpu_batch_destroy": ([C.c_void_p], C.c_int),
    "dimgpu_batch_last_error": ([C.c_void_p], C.c_char_p),
    "dimgpu_batch_add": ([C.c_void_p, _D, _DP, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_int)], C.c_int),
    "dimgpu_batch_remove": ([C.c_void_p, C.c_int], C.c_int),
    "dimgpu_batch_run": ([C.c_void_p, C.c_int], C.c_int),
    "dimgpu_batch_status": ([C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "dimgpu_batch_download": ([C.c_void_p, C.c_int, _DP, C.c_size_t, _DP], C.c_int),
    "dimgpu_batch_set_grid": ([C.c_void_p, C.c_int], C.c_int),
    "dimgpu_batch_size": ([C.c_void_p], C.c_int),
    "dimgpu_batch_set_stream": ([C.c_void_p, C.c_void_p], C.c_int),
    "dimgpu_advance_one_step": ([_D, _DP, _DP, C.c_double, C.c_double, _DP,
                                 C.POINTER(abi.PhaseTimes)], C.c_int),
    "dimgpu_batch_reserve": ([C.c_void_p, C.c_longlong, C.c_int, C.c_longlong], C.c_int),
    "dimgpu_batch_arena_used": ([C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)], C.c_int),
    "dimgpu_batch_enqueue": ([C.c_void_p, C.c_int], C.c_int),
    "dimgpu_batch_wait": ([C.c_void_p], C.c_int),
    "dimgpu_init_shock_bubble": ([_S, C.POINTER(abi.ShockBubbleIC)], C.c_int),
    "dimgpu_init_bubble_cloud": ([_S, C.POINTER(abi.BubbleCloudIC), C.POINTER(abi.BubbleIC), C.c_int], C.c_int),
    "dimgpu_csv_write_async": ([_S, C.c_char_p, _DP, _DP, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "dimgpu_csv_wait": ([C.c_void_p], C.c_int),
    "dimgpu_slabs_create": ([_D, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_void_p)], C.c_int),
    "dimgpu_slabs_destroy": ([C.c_void_p], C.c_int),
    "dimgpu_slabs_last_error": ([C.c_void_p], C.c_char_p),
    "dimgpu_slabs_upload": ([C.c_void_p, _DP, C.c_size_t], C.c_int),
    "dimgpu_slabs_step": ([C.c_void_p, C.c_double, C.c_double, _DP], C.c_int),
    "dimgpu_slabs_download": ([C.c_void_p, _DP, C.c_size_t], C.c_int),
    "dimgpu_server_create": ([C.POINTER(abi.ServerConfig), C.POINTER(C.c_void_p)], C.c_int),
    "dimgpu_server_destroy": ([C.c_void_p], C.c_int),
    "dimgpu_server_last_error": ([C.c_void_p], C.c_char_p),
    "dimgpu_server_submit": ([C.c_void_p, _D, _DP, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_longlong)],
                             C.c_int),
    "dimgpu_server_poll": ([C.c_void_p, C.c_longlong, C.POINTER(C.c_int), _DP, C.c_size_t, _DP,
                           C.POINTER(C.c_double)], C.c_int),
    "dimgpu_server_cancel": ([C.c_void_p, C.c_longlong], C.c_int),
    "dimgpu_server_drain": ([C.c_void_p], C.c_int),
    "dimgpu_server_stats": ([C.c_void_p, C.POINTER(abi.ServerCounters)], C.c_int),
}

_lib = None


class DimGpuError(RuntimeError):
    """A non-zero dimgpu status; .status holds the code (abi.E_*)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def lib() -> C.CDLL:
    """The loaded library (loads it on first use; raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run python -m diffuse_vs_gfm_mms_b200.build")
        L = C.CDLL(LIB_PATH)
        for name, (argtypes, restype) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = argtypes
            f.restype = restype
        _lib = L
    return _lib


def check(rc: int, session=None) -> None:
    if rc != 0:
        msg = lib().dimgpu_last_error(session)
        raise DimGpuError(rc, msg.decode() if msg else "")
