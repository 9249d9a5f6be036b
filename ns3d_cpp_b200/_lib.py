"""Loader of the native library ``libns3d_b200.so`` with ctypes signatures.

The library is built in-tree by :mod:`ns3d_cpp_b200.build`. If it is missing or
older than its sources, :func:`load` builds it (nvcc is required); if that is
impossible it raises -- there is no pure-Python or CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re
import threading

from . import build as _build

_LIB = None
_LOCK = threading.Lock()

HEADER = os.path.join(_build.INCLUDE, "ns3d_gpu.h")

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_D = ctypes.POINTER(ctypes.c_double)
_pvp = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); ns3d_params* / ns3d_turb_stats* passed as c_void_p
_SIGS = {
    "ns3d_params_default": (_i, [_vp]),
    "ns3d_params_from_file": (_i, [ctypes.c_char_p, _vp]),
    "ns3d_params_derive": (_i, [_vp]),
    "ns3d_params_size": (ctypes.c_size_t, []),
    "ns3d_turb_stats_size": (ctypes.c_size_t, []),
    "ns3d_create": (_i, [_vp, _i, _pvp]),
    "ns3d_destroy": (_i, [_vp]),
    "ns3d_last_error": (ctypes.c_char_p, [_vp]),
    "ns3d_get_params": (_i, [_vp, _vp]),
    "ns3d_device_bytes": (_i, [_vp, ctypes.POINTER(ctypes.c_size_t)]),
    "ns3d_synchronize": (_i, [_vp]),
    "ns3d_upload_primitive": (_i, [_vp, _D, _D, _D, _D, _D, _i]),
    "ns3d_prefetch_primitive": (_i, [_vp, _D, _D, _D, _D, _D, _i]),
    "ns3d_upload_conserved": (_i, [_vp, _D, _D, _D, _D, _D, _i]),
    "ns3d_download_primitive": (_i, [_vp, _D, _D, _D, _D, _D, _D, _D, _i]),
    "ns3d_download_conserved": (_i, [_vp, _D, _D, _D, _D, _D, _i]),
    "ns3d_record_conserved0": (_i, [_vp]),
    "ns3d_compute_rhs": (_i, [_vp, _D, _D, _D, _D, _D, _i]),
    "ns3d_compute_timestep": (_i, [_vp, _D]),
    "ns3d_runge_kutta_3": (_i, [_vp, _d]),
    "ns3d_time_advance": (_i, [_vp, _i, _D, ctypes.POINTER(ctypes.c_int)]),
    "ns3d_step": (_i, [_vp, _i]),
    "ns3d_last_dt": (_i, [_vp, _D]),
    "ns3d_step_times": (_i, [_vp, _D, _i, ctypes.POINTER(ctypes.c_int)]),
    "ns3d_total_energy": (_i, [_vp, _D]),
    "ns3d_energy_spectrum": (_i, [_vp, _D, _i]),
    "ns3d_turbulence_stats": (_i, [_vp, _vp]),
    "ns3d_init_isotropic": (_i, [_vp, _i, ctypes.c_double, ctypes.c_ulonglong, ctypes.c_double]),
    "ns3d_tecplot_write": (_i, [_vp, _D, _D, _D, _D, _D, ctypes.c_char_p, ctypes.c_double, _i]),
    "ns3d_tecplot_read": (_i, [_vp, ctypes.c_char_p, _D, _D, _D, _D, _D]),
    "ns3d_tecplot_read_downsample": (_i, [_vp, ctypes.c_char_p, _i, _i, _i, _D, _D, _D, _D, _D]),
    "ns3d_write_tecplot": (_i, [_vp, ctypes.c_char_p, ctypes.c_double]),
    "ns3d_residuals": (_i, [_vp, _D]),
    "ns3d_time_advance_segment": (_i, [_vp, _i, _D, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    "ns3d_turbulence_stats_spectrum": (_i, [_vp, _D, _i, _vp]),
    "ns3d_spectrum_write": (_i, [ctypes.c_char_p, _D, _i]),
    "ns3d_stats_write": (_i, [ctypes.c_char_p, ctypes.c_double, _vp]),
    "ns3d_run": (_i, [_vp, ctypes.c_char_p, _i, _i, _D, ctypes.POINTER(ctypes.c_int)]),
    "ns3d_checkpoint_write": (_i, [_vp, ctypes.c_char_p]),
    "ns3d_checkpoint_read": (_i, [_vp, ctypes.c_char_p]),
    "ns3d_checkpoint_check": (_i, [ctypes.c_char_p, _vp]),
    "ns3d_completed_steps": (_i, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "ns3d_residuals_write": (_i, [ctypes.c_char_p, _i, _D, ctypes.c_double]),
    "ns3d_read_tecplot": (_i, [_vp, ctypes.c_char_p]),
    "ns3d_get_stream": (_i, [_vp, _pvp]),
    "ns3d_profile": (_i, [_vp, _i]),
    "ns3d_profile_read": (_i, [_vp, _D, ctypes.POINTER(ctypes.c_longlong)]),
    "ns3d_launch_count": (_i, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "ns3d_rhs_vjp": (_i, [_vp, _D, _D]),
    "ns3d_step_dts": (_i, [_vp, _i, _D]),
    "ns3d_adjoint": (_i, [_vp, _i, _i, _D, _D, _D, _D, _D]),
    # device pointers and the stream passed as integers (c_void_p)
    "ns3d_compute_rhs_noalloc": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
}


def header_functions(path: str = HEADER) -> list[str]:
    """Names of the functions include/ns3d_gpu.h declares."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ns3d_[a-z0-9_]+)\s*\(", text)))


def library_path() -> str:
    return _build.LIB


def load(build_if_needed: bool = True) -> ctypes.CDLL:
    global _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        if build_if_needed and _build.needs_build():
            _build.build()
        if not os.path.exists(_build.LIB):
            raise RuntimeError(f"native library missing: {_build.LIB} (run ns3d_cpp_b200.build)")
        lib = ctypes.CDLL(_build.LIB)
        for name, (res, args) in _SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _LIB = lib
        from .solver import SolverParams, TurbStats  # layout check against the C structs
        if lib.ns3d_params_size() != ctypes.sizeof(SolverParams):
            raise RuntimeError("ns3d_params layout mismatch between C and Python")
        if lib.ns3d_turb_stats_size() != ctypes.sizeof(TurbStats):
            raise RuntimeError("ns3d_turb_stats layout mismatch between C and Python")
        return lib
