"""ctypes bindings of libpyrocmc.so (include/pyrocmc.h).

The library is the only compute path: if it cannot be loaded, or no CUDA
device is present when a system is created, the calls fail loudly. There is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

_lib = None

_I = C.c_int
_D = C.c_double
_U64 = C.c_uint64
_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
_U64P = C.POINTER(C.c_uint64)
_IP = C.POINTER(C.c_int)
_CPP = C.POINTER(C.c_char_p)

_SIGNATURES = {
    "pc_last_error": (C.c_char_p, []),
    "pc_version": (_I, []),
    "pc_pyrochlore_displacements": (_I, [_I, _I, _I64P, _I, _IP]),
    "pc_create": (_I, [_I, _I32P, _U64, _PP]),
    "pc_destroy": (_I, [_P]),
    "pc_set_stream": (_I, [_P, _P]),
    "pc_set_seed": (_I, [_P, _U64]),
    "pc_define_coupling": (_I, [_P, C.c_char_p, _I64P, _I32P, _DP]),
    "pc_set_coupling_matrix": (_I, [_P, _I, _DP]),
    "pc_set_coupling_matrices": (_I, [_P, _I, _IP, _DP]),
    "pc_energy_device": (_I, [_P, _P]),
    "pc_energy_groups_device": (_I, [_P, _P, _P]),
    "pc_energy_grad_device": (_I, [_P, _P, _P, _P, _I]),
    "pc_set_global_field": (_I, [_P, _DP]),
    "pc_get_global_field": (_I, [_P, _DP]),
    "pc_set_T_ref": (_I, [_P, _D]),
    "pc_set_overrelax_mode": (_I, [_P, _I]),
    "pc_set_colouring": (_I, [_P, _I]),
    "pc_set_kernel_path": (_I, [_P, _I]),
    "pc_set_sweep_schedule": (_I, [_P, _I]),
    "pc_set_update": (_I, [_P, _I]),
    "pc_ssf_set_resolved": (_I, [_P, _I]),
    "pc_lt_minimum": (_I, [_I, _D, _D, _D, _D, _DP, _DP, _I64P, _DP]),
    "pc_ssf_merge": (_I, [_P, _I32P, _I, _DP, _DP, _DP, _DP, _DP, _DP, _DP]),
    "pc_kernel_path": (_I, [_P, _IP]),
    "pc_setup_lattice": (_I, [_P]),
    "pc_num_replicas": (_I, [_P, _IP]),
    "pc_num_spins": (_I, [_P, _I, _I64P]),
    "pc_colours": (_I, [_P, _IP, _I32P]),
    "pc_neighbour_table": (_I, [_P, _I, _I, _I, _I32P]),
    "pc_site_positions": (_I, [_P, _I, _I64P, _I32P]),
    "pc_launch_count": (_I, [_P, _U64P]),
    "pc_set_spins": (_I, [_P, _I, _DP]),
    "pc_get_spins": (_I, [_P, _I, _DP]),
    "pc_set_spins_f4": (_I, [_P, _I, _FP]),
    "pc_get_spins_f4": (_I, [_P, _I, _FP]),
    "pc_random_spins": (_I, [_P, _U64]),
    "pc_spins_device": (_I, [_P, _I, _PP]),
    "pc_get_sweep_counter": (_I, [_P, _I, _U64P]),
    "pc_set_sweep_counter": (_I, [_P, _I, _U64]),
    "pc_sweep": (_I, [_P, _DP, _I, _I, _U64P]),
    "pc_overrelax_all": (_I, [_P]),
    "pc_overrelax_theta": (_I, [_P, _I, _DP]),
    "pc_energy": (_I, [_P, _DP, _DP]),
    "pc_local_field": (_I, [_P, _I, _DP]),
    "pc_ssf_configure": (_I, [_P, _CPP, _I, _I, _I32P]),
    "pc_ssf_sample": (_I, [_P, _I32P]),
    "pc_ssf_read": (_I, [_P, _I, _DP, _DP, _U64P]),
    "pc_ssf_clear": (_I, [_P, _I]),
    "pc_ssf_current": (_I, [_P, _I, _DP]),
    "pc_pt_configure": (_I, [_P, _DP]),
    "pc_pt_run": (_I, [_P, _I, _I, _I]),
    "pc_pt_reset_stats": (_I, [_P]),
    "pc_pt_read_energy": (_I, [_P, _DP, _DP, _DP, _U64P]),
    "pc_pt_read_exchange": (_I, [_P, _U64P, _U64P]),
    "pc_pt_slots": (_I, [_P, _I32P]),
    "pc_energy_grad": (_I, [_P, _DP, _DP, _P, _DP, _DP]),
    "pc_energy_grad_field": (_I, [_P, _P, _DP, _DP, _P, _DP, _DP]),
    "pc_set_wait_limit": (_I, [_P, _I]),
    "pc_spin_ft": (_I, [_P, _I, _DP]),
    "pc_ssf_forward": (_I, [_P, _P]),
    "pc_ssf_backward": (_I, [_P, _P, _P]),
    "pc_ssf_forward_keep": (_I, [_P, _P, C.POINTER(C.c_uint64)]),
    "pc_ssf_backward_kept": (_I, [_P, C.c_uint64, _P, _P]),
    "pc_energy_noalloc": (_I, [_P, _I, _DP, _P, _P]),
    "pc_autotune": (_I, [_P]),
    "pc_set_load_variant": (_I, [_P, _I]),
    "pc_get_load_variant": (_I, [_P, _IP]),
    "pc_get_tile": (_I, [_P, _IP, _IP]),
    "pc_set_tile": (_I, [_P, _I, _I]),
    "pc_step_host": (_I, [_P, _FP, _FP, _D, _I, _I, _I, _DP, _U64P]),
    "pc_step_host3": (_I, [_P, _FP, _FP, _D, _I, _I, _I, _DP, _U64P]),
    "pc_last_kernel_times": (_I, [_P, _DP, _DP]),
    "pc_set_kernel_timing": (_I, [_P, _I]),
    "pc_set_launch_overlap": (_I, [_P, _I]),
    "pc_set_cluster_sweeps": (_I, [_P, _I]),
    "pc_get_cluster_sweeps": (_I, [_P, _IP]),
    "pc_set_pt_persistent": (_I, [_P, _I]),
    "pc_get_pt_persistent": (_I, [_P, _IP]),
}


class PyroCMCError(RuntimeError):
    """Raised when a libpyrocmc call returns a nonzero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[pc error {code}] {message}")
        self.code = code


class InvalidArgument(PyroCMCError, ValueError):
    pass


ERR_INVALID, ERR_CUDA, ERR_STATE, ERR_UNSUPPORTED, ERR_TIMEOUT = 1, 2, 3, 4, 5


def lib_path() -> str:
    return _build.LIB


def lib():
    """Loads libpyrocmc.so, building it with nvcc first if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(_build.LIB):
            _build.build()
        l = C.CDLL(_build.LIB)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        msg = lib().pc_last_error().decode(errors="replace")
        if rc == ERR_INVALID:
            raise InvalidArgument(rc, msg)
        raise PyroCMCError(rc, msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))
