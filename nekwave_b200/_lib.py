"""ctypes binding of libnwb (include/nwb.h).

The shared library is built in-tree (``nekwave_b200/libnwb.so``, see
``nekwave_b200/csrc/Makefile``).  There is no fallback: if the library is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnwb.so")

NWB_OK = 0
NWB_EINVAL = 1
NWB_ENOMEM = 2
NWB_ECUDA = 3
NWB_ETIMEOUT = 4
NWB_ENONFINITE = 5
NWB_EBUSY = 6
NWB_ENOTFOUND = 7

NWB_FP64 = 0
NWB_FP32_BULK = 1
NWB_SOLVER_TRUE_PMC = 1  # nwb_solver_create_ex flag

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


class NwbError(RuntimeError):
    """A libnwb call returned a status other than NWB_OK."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_status_name(status)}: {message}")
        self.status = status


class MeshDesc(C.Structure):
    """nwb_mesh_desc (include/nwb.h)."""
    _fields_ = [("N", C.c_int), ("nelt", C.c_int), ("D", _D), ("w3", _D), ("jac", _D),
                ("met", _D * 9), ("vol_idx_minus", _I), ("vol_idx_plus", _I),
                ("bc_type", _I), ("nx", _D), ("ny", _D), ("nz", _D), ("dA", _D)]


class SolverInfo(C.Structure):
    """nwb_solver_info (include/nwb.h)."""
    _fields_ = [("N", C.c_int), ("nelt", C.c_int), ("npts", C.c_longlong),
                ("stride", C.c_longlong), ("geometry", C.c_int), ("precision", C.c_int),
                ("ks", C.c_int), ("epb", C.c_int), ("threads_per_block", C.c_int),
                ("smem_bytes", C.c_int), ("device_bytes", C.c_longlong), ("ksmem", C.c_int),
                ("minb", C.c_int), ("variant", C.c_int), ("variant_count", C.c_int),
                ("structured", C.c_int * 3), ("periodic_mask", C.c_int)]


# name -> (restype, argtypes); every symbol include/nwb.h declares.
SIGNATURES = {
    "nwb_last_error": (C.c_char_p, []),
    "nwb_status_string": (C.c_char_p, [C.c_int]),
    "nwb_version": (C.c_int, []),
    "nwb_set_device": (C.c_int, [C.c_int]),
    "nwb_box_mesh_create": (C.c_int, [C.c_int] * 4 + [C.c_double] * 6 +
                            [C.c_int, C.POINTER(C.c_void_p)]),
    "nwb_box_mesh_desc": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc)]),
    "nwb_box_mesh_coords": (C.c_int, [C.c_void_p] + [C.POINTER(_D)] * 3),
    "nwb_box_mesh_gll": (C.c_int, [C.c_void_p] + [C.POINTER(_D)] * 2),
    "nwb_box_mesh_dxmin": (C.c_int, [C.c_void_p, _D]),
    "nwb_box_mesh_destroy": (None, [C.c_void_p]),
    "nwb_box_probes": (C.c_int, [C.c_int] * 4 + [C.c_double] * 6 + [C.c_int, _D, _I, _D]),
    "nwb_solver_create": (C.c_int, [C.POINTER(MeshDesc), C.c_double, C.c_int,
                                    C.POINTER(C.c_void_p)]),
    "nwb_solver_create_ex": (C.c_int, [C.POINTER(MeshDesc), C.c_double, C.c_int, C.c_uint,
                                       C.POINTER(C.c_void_p)]),
    "nwb_solver_create_box": (C.c_int, [C.c_int] * 4 + [C.c_double] * 6 +
                              [C.c_int, C.c_double, C.c_int, C.POINTER(C.c_void_p)]),
    "nwb_solver_init_pulse": (C.c_int, [C.c_void_p, _D]),
    "nwb_upload_state": (C.c_int, [C.c_void_p, _D, C.c_size_t]),
    "nwb_download_state": (C.c_int, [C.c_void_p, _D, C.c_size_t]),
    "nwb_download_nodes": (C.c_int, [C.c_void_p, C.c_longlong, C.c_longlong, _D, C.c_size_t]),
    "nwb_step": (C.c_int, [C.c_void_p, C.c_double, C.c_int]),
    "nwb_sync": (C.c_int, [C.c_void_p]),
    "nwb_eval_rhs": (C.c_int, [C.c_void_p, _D, C.c_size_t]),
    "nwb_energy": (C.c_int, [C.c_void_p, _D]),
    "nwb_max_norms": (C.c_int, [C.c_void_p, _D, _D]),
    "nwb_probe_setup": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_longlong), _D]),
    "nwb_probe_read": (C.c_int, [C.c_void_p, _D]),
    "nwb_snapshot_begin": (C.c_int, [C.c_void_p, _D, C.c_size_t]),
    "nwb_snapshot_wait": (C.c_int, [C.c_void_p]),
    "nwb_upload_begin": (C.c_int, [C.c_void_p, _D, C.c_size_t]),
    "nwb_upload_wait": (C.c_int, [C.c_void_p]),
    "nwb_solver_destroy": (C.c_int, [C.c_void_p]),
    "nwb_solver_get_info": (C.c_int, [C.c_void_p, C.POINTER(SolverInfo)]),
    "nwb_solver_device_state": (C.c_int, [C.c_void_p, C.POINTER(_D), C.POINTER(C.c_void_p)]),
    "nwb_solver_launch_count": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "nwb_energy_noalloc": (C.c_int, [_D, C.c_longlong, C.c_int, C.c_int, _D, C.c_int, _D, _D,
                                     C.c_void_p]),
    "nwb_solver_set_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "nwb_solver_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_float), C.c_int]),
    "nwb_pool_create": (C.c_int, [C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "nwb_pool_add": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.c_double, C.c_double, C.c_int,
                               C.c_int, _I, _D, C.c_int, C.POINTER(C.c_int)]),
    "nwb_pool_add_box": (C.c_int, [C.c_void_p] + [C.c_int] * 4 + [C.c_double] * 6 +
                         [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _D, C.c_int,
                          C.POINTER(C.c_int)]),
    "nwb_pool_init_pulse": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "nwb_pool_upload": (C.c_int, [C.c_void_p, C.c_int, _D, C.c_size_t]),
    "nwb_pool_step": (C.c_int, [C.c_void_p, C.c_int]),
    "nwb_pool_sync": (C.c_int, [C.c_void_p]),
    "nwb_pool_query": (C.c_int, [C.c_void_p, _I, _I, C.c_int]),
    "nwb_pool_results": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D]),
    "nwb_pool_query_begin": (C.c_int, [C.c_void_p]),
    "nwb_pool_query_end": (C.c_int, [C.c_void_p, _I, _I, C.c_int]),
    "nwb_pool_results_async": (C.c_int, [C.c_void_p, C.c_int, _D, _D, _D]),
    "nwb_pool_remove": (C.c_int, [C.c_void_p, C.c_int]),
    "nwb_pool_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                _I, C.POINTER(C.c_longlong)]),
    "nwb_pool_time_steps": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float)]),
    "nwb_pool_set_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "nwb_pool_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "nwb_pool_destroy": (C.c_int, [C.c_void_p]),
    "nwb_time_steps": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int,
                                 C.POINTER(C.c_float)]),
    "nwb_time_stage_kernel": (C.c_int, [C.c_void_p, C.c_double, C.c_int,
                                        C.POINTER(C.c_float)]),
}

_lib = None


def _status_name(status: int) -> str:
    names = {0: "NWB_OK", 1: "NWB_EINVAL", 2: "NWB_ENOMEM", 3: "NWB_ECUDA",
             4: "NWB_ETIMEOUT", 5: "NWB_ENONFINITE", 6: "NWB_EBUSY", 7: "NWB_ENOTFOUND"}
    return names.get(status, f"status {status}")


def lib() -> C.CDLL:
    """Load libnwb.so once; raise if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libnwb.so not built ({LIB_PATH}); run `make -C nekwave_b200/csrc` "
                "or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != NWB_OK:
        msg = lib().nwb_last_error()
        raise NwbError(status, msg.decode() if msg else "")


def dptr(a):
    return a.ctypes.data_as(_D)


def iptr(a):
    return a.ctypes.data_as(_I)
