"""ctypes binding of librr_b200.so (the C ABI declared in include/rr_rank.h).

The library is the product: there is no CPU fallback.  If the shared object
is missing, loading raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librr_b200.so")

RR_OK = 0
STATUS_NAMES = {0: "RR_OK", 1: "RR_EINVAL", 2: "RR_EPRIME", 3: "RR_ENOMEM", 4: "RR_ECUDA", 5: "RR_ETIMEOUT",
                6: "RR_EIO", 7: "RR_ESTATE", 8: "RR_EUNSUPPORTED"}

# Every symbol include/rr_rank.h declares, with (restype, argtypes).
_vp = C.c_void_p
_i32, _i64, _u32 = C.c_int32, C.c_int64, C.c_uint32
_pi64, _pu32, _pi32 = C.POINTER(C.c_int64), C.POINTER(C.c_uint32), C.POINTER(C.c_int32)
# rr_progress_fn: int (*)(void* user, int64_t len, int64_t target_len, double elapsed_s, double terms_per_s)
PROGRESS_FN = C.CFUNCTYPE(C.c_int, _vp, _i64, _i64, C.c_double, C.c_double)
SIGNATURES = {
    "rr_status_string": (C.c_char_p, [C.c_int]),
    "rr_last_error": (C.c_char_p, []),
    "rr_version": (C.c_char_p, []),
    "rr_ctx_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "rr_ctx_destroy": (C.c_int, [_vp]),
    "rr_ctx_stream": (_vp, [_vp]),
    "rr_ctx_synchronize": (C.c_int, [_vp]),
    "rr_ctx_set_pm_tensor_cores": (C.c_int, [_vp, _i32]),
    "rr_prime_check": (C.c_int, [_u32]),
    "rr_matrix_create": (C.c_int, [_vp, _i64, _i64, _vp, _vp, _vp, _u32, C.POINTER(_vp)]),
    "rr_matrix_destroy": (C.c_int, [_vp]),
    "rr_matrix_max_nnzs": (C.c_int, [_vp, _pi64, _pi64]),
    "rr_matrix_shape": (C.c_int, [_vp, _pi64, _pi64, _pi64]),
    "rr_krylov_create": (C.c_int, [_vp, _i32, _vp, _vp, _vp, _i64, C.POINTER(_vp)]),
    "rr_krylov_destroy": (C.c_int, [_vp]),
    "rr_krylov_advance": (C.c_int, [_vp, _i64, _vp, _i64, _pi64]),
    "rr_krylov_advance_report": (C.c_int, [_vp, _i64, _vp, _i64, _i64, PROGRESS_FN, _vp, _pi64]),
    "rr_krylov_fill_status": (C.c_int, [_vp, C.c_char_p, _i64]),
    "rr_krylov_step_device": (C.c_int, [_vp, _i64]),
    "rr_krylov_fetch": (C.c_int, [_vp, _i64, _i64, _vp, _i64]),
    "rr_krylov_length": (C.c_int, [_vp, _pi64]),
    "rr_krylov_get_curv": (C.c_int, [_vp, _vp]),
    "rr_krylov_bytes_per_application": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "rr_krylov_phase_bytes": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "rr_krylov_profile": (C.c_int, [_vp, _i64, C.POINTER(C.c_double)]),
    "rr_krylov_launch_count": (C.c_int, [_vp, _pi64]),
    "rr_pm_basis": (C.c_int, [_vp, _vp, _i64, _i32, _i64, _i64, _u32, _vp, _vp]),
    "rr_pm_basis_short_noalloc": (C.c_int, [_vp, _i64, _i32, _i64, _i64, _u32, _vp, _vp, _vp]),
    "rr_rank_from_basis": (C.c_int, [_vp, _vp, _i32, _i64, _u32, _pi64]),
    "rr_is_generating_poly": (C.c_int, [_vp, _i64, _vp, _i64, _i32, _u32, C.POINTER(C.c_int32)]),
    "rr_berlekamp_massey": (C.c_int, [_vp, _i64, _u32, _vp, _pi64]),
    "rr_pm_basis_batch": (C.c_int, [_vp, _i32, _vp, _vp, _i32, _i64, _i64, _u32, _vp, _vp]),
    "rr_rank": (C.c_int, [_vp, _i32, _vp, _vp, _vp, _i64, _pi64]),
    "rr_batch_create": (C.c_int, [_vp, _i32, _vp, _vp, _vp, _vp, _vp, _u32, _i32, _vp, _vp, _vp, C.POINTER(_vp)]),
    "rr_batch_destroy": (C.c_int, [_vp]),
    "rr_batch_krylov": (C.c_int, [_vp]),
    "rr_batch_sequence": (C.c_int, [_vp, _i32, _vp, _i64, _pi64]),
    "rr_batch_ranks": (C.c_int, [_vp, _i32, _vp]),
    "rr_batch_info": (C.c_int, [_vp, _pi64, _pi64, _pi64, _pi64]),
    "rr_batch_tuning": (C.c_int, [_vp, _pi32, _vp, _vp]),
    "rr_batch_tuning_shape": (C.c_int, [_vp, _pi32, _vp, _vp]),
    "rr_device_barrier_check": (C.c_int, [_vp, _i32, _i32, _i32, C.c_double, _pi32]),
    "rr_wdm_save": (C.c_int, [C.c_char_p, _i64, _i64, _u32, _i32, _vp, _vp, _vp, _vp, _vp, _i64, _i64]),
    "rr_wdm_load": (C.c_int, [C.c_char_p, _pi64, _pi64, _pu32, _pi32, _pi64, _vp, _vp, _vp, _vp, _vp, _i64]),
    "rr_sms_load": (C.c_int, [C.c_char_p, _u32, _pi64, _pi64, _pi64, _vp, _vp, _vp]),
    "rr_server_create": (C.c_int, [C.c_int, _vp, C.POINTER(_vp)]),
    "rr_server_submit": (C.c_int, [_vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(C.c_uint64)]),
    "rr_server_wait": (C.c_int, [_vp, C.c_uint64, C.c_double, _pi64, C.POINTER(C.c_double)]),
    "rr_server_stats": (C.c_int, [_vp, _pi64, _pi64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]),
    "rr_server_destroy": (C.c_int, [_vp]),
    "rr_footprint": (C.c_int, [_i64, _i64, _i64, _i32, C.POINTER(C.c_uint64)]),
    "rr_place_by_footprint": (C.c_int, [_i32, _vp, _i32, _vp, _vp, _vp]),
    "rr_fleet_create": (C.c_int, [_vp, _i32, _vp, C.POINTER(_vp)]),
    "rr_fleet_submit": (C.c_int, [_vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _vp, C.POINTER(C.c_uint64)]),
    "rr_fleet_wait": (C.c_int, [_vp, C.c_uint64, C.c_double, _pi64, C.POINTER(C.c_double)]),
    "rr_fleet_device_of": (C.c_int, [_vp, C.c_uint64, _pi32]),
    "rr_fleet_stats": (C.c_int, [_vp, _pi64, _pi64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]),
    "rr_fleet_destroy": (C.c_int, [_vp]),
    "rr_batch_ranks_multi": (C.c_int, [_vp, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _u32, _i32, _vp, _vp, _vp, _i32,
                                       _vp, _vp]),
}


class ServerConfig(C.Structure):
    """rr_server_config of include/rr_rank.h."""

    _fields_ = [("b", C.c_int32), ("p", C.c_uint32), ("lanes", C.c_int32), ("workers", C.c_int32),
                ("max_active", C.c_int32), ("chunk_apps", C.c_int64), ("hbm_budget", C.c_uint64)]

_LIB = None


class RRError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} not built: run `make -C rust_rank_b200/csrc` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def check(status: int) -> None:
    if status != RR_OK:
        msg = lib().rr_last_error().decode(errors="replace")
        raise RRError(status, msg)


def ptr(a: np.ndarray):
    """Data pointer of a C-contiguous numpy array (None for None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)
