"""Loader of libmgfvm.so (the CUDA engine and its C ABI, include/mgfvm.h).

There is no fallback: if the library is missing or fails to load, every entry point
of this package raises.  Build it with `make -C multigrid-fvm_b200` (or
`python __graft_entry__.py build` at the repository root).
"""
from __future__ import annotations

import ctypes as C
import os

from . import _abi

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MGFVM_LIB", os.path.join(os.path.dirname(PKG), "lib", "libmgfvm.so"))

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


class MgfvmError(RuntimeError):
    """A C-ABI call returned a non-OK status."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libmgfvm.so not found at {LIB_PATH}; build it with "
                          f"`make -C {os.path.dirname(PKG)}`")
    L = C.CDLL(LIB_PATH)
    sig = {
        "mgfvm_config_default": (None, [C.POINTER(_abi.Config)]),
        "mgfvm_options_default": (None, [C.POINTER(_abi.Options)]),
        "mgfvm_config_read": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_abi.Config), C.c_int]),
        "mgfvm_config_release": (None, [C.POINTER(_abi.Config)]),
        "mgfvm_config_validate": (C.c_int, [C.POINTER(_abi.Config)]),
        "mgfvm_create": (C.c_int, [C.POINTER(_abi.Config), C.c_int, C.POINTER(_abi.Options), C.POINTER(_vp)]),
        "mgfvm_destroy": (C.c_int, [_vp]),
        "mgfvm_reset": (C.c_int, [_vp]),
        "mgfvm_set_inlet_profile": (C.c_int, [_vp, C.c_int, _dp, C.c_int]),
        "mgfvm_cycle": (C.c_int, [_vp, C.c_int]),
        "mgfvm_solve": (C.c_int, [_vp, C.c_int, C.c_double, _ip]),
        "mgfvm_history": (C.c_int, [_vp, C.c_int, _dp, _dp, C.c_int, _ip]),
        "mgfvm_num_levels": (C.c_int, [_vp, C.c_int, _ip]),
        "mgfvm_level_dims": (C.c_int, [_vp, C.c_int, C.c_int, _ip, _ip]),
        "mgfvm_get_field": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp]),
        "mgfvm_set_field": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp]),
        "mgfvm_get_tag": (C.c_int, [_vp, C.c_int, C.c_int, _ip]),
        "mgfvm_get_obstacle_ranges": (C.c_int, [_vp, C.c_int, C.c_int, _ip]),
        "mgfvm_op": (C.c_int, [_vp, C.c_int, C.c_int]),
        "mgfvm_kernel_launches": (C.c_int, [_vp, C.POINTER(C.c_longlong)]),
        "mgfvm_last_elapsed_ms": (C.c_int, [_vp, _dp]),
        "mgfvm_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
        "mgfvm_time_op": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, _ip]),
        "mgfvm_profile_cycle": (C.c_int, [_vp, _dp, _ip, _ip, C.c_int, _ip]),
        "mgfvm_get_tuning": (C.c_int, [_vp, C.POINTER(_abi.Tuning)]),
        "mgfvm_set_tuning": (C.c_int, [_vp, C.POINTER(_abi.Tuning)]),
        "mgfvm_autotune": (C.c_int, [_vp, C.c_int, C.POINTER(_abi.Tuning), _dp, _dp]),
        "mgfvm_transfer_bytes": (C.c_int, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
        "mgfvm_last_error": (C.c_char_p, []),
        "mgfvm_pattern_staggered": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                               C.c_ulonglong, _ip]),
        "mgfvm_pattern_random": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                            C.c_ulonglong, _ip, _ip, C.c_int, _ip]),
        "mgfvm_pattern_pixels": (C.c_int, [_ip, C.c_int, _ip, C.c_int, _ip]),
        "mgfvm_write_vtk": (C.c_int, [C.c_char_p, C.POINTER(_abi.Config), C.c_int, C.c_int, _dp, _dp, _dp,
                                       _dp, _ip, C.c_int, _dp]),
        "mgfvm_write_convergence": (C.c_int, [C.c_char_p, _dp, C.c_int, C.c_int, C.c_int]),
        "mgfvm_jacobi_f64": (C.c_int, [_vp] * 8 + [C.c_int] * 5 + [_vp]),
        "mgfvm_rbgs_f64": (C.c_int, [_vp] * 7 + [C.c_int] * 5 + [_vp]),
        "mgfvm_masserror_f64": (C.c_int, [_vp] * 6 + [C.c_int, C.c_int, _vp, _vp, _vp]),
        "mgfvm_masserror_scratch_doubles": (C.c_size_t, [C.c_int, C.c_int]),
        "mgfvm_masserror_f64_noalloc": (C.c_int, [_vp] * 6 + [C.c_int, C.c_int, _vp, _vp]),
        "mgfvm_check_division": (C.c_int, [C.c_int, C.c_longlong, C.c_ulonglong, _vp]),
        "mgfvm_field_device_ptr": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p), _ip, _ip]),
        "mgfvm_set_direction": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
        "mgfvm_get_tangent": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp]),
        "mgfvm_objective": (C.c_int, [_vp, C.c_int, _dp, _dp]),
        "mgfvm_gradient": (C.c_int, [C.POINTER(_abi.Config), _dp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp]),
        "mgfvm_adjoint": (C.c_int, [_vp, C.c_int]),
        "mgfvm_adjoint_gradient": (C.c_int, [_vp, C.c_int, _dp, _dp, _dp, _dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != _abi.OK:
        msg = lib().mgfvm_last_error()
        raise MgfvmError(status, msg.decode() if msg else "")


def exported_symbols():
    """Every function include/mgfvm.h declares (used by the load test)."""
    hdr = os.path.join(os.path.dirname(os.path.dirname(PKG)), "include", "mgfvm.h")
    import re
    names = []
    with open(hdr) as f:
        text = f.read()
    for m in re.finditer(r"^\s*(?:const\s+)?[a-z_ ]+\**\s*\**(mgfvm_[a-z0-9_]+)\s*\(", text, re.M):
        names.append(m.group(1))
    return sorted(set(names))
