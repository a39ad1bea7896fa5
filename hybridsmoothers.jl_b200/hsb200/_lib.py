"""ctypes binding of libhsb200.so (the C ABI declared in include/hsb200.h).

The library is the only compute path: if it is missing, importing a compute
entry point raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhsb200.so")

HS_OK, HS_ERR_ARG, HS_ERR_OOM, HS_ERR_CUDA, HS_ERR_SINGULAR = 0, 1, 2, 3, 4
HS_ERR_NONFINITE, HS_ERR_NOT_CONVERGED, HS_ERR_TIMEOUT, HS_ERR_UNSUPPORTED, HS_ERR_BUDGET = 5, 6, 7, 8, 9
HS_F64, HS_F32 = 0, 1
HS_CSC, HS_CSR = 0, 1
HS_SWEEP_FORWARD, HS_SWEEP_BACKWARD, HS_SWEEP_SYMMETRIC = 0, 1, 2
HS_CACHE_PACKED, HS_CACHE_VIEW = 0, 1
HS_EIG_POWER, HS_EIG_LANCZOS = 0, 1
HS_PREC_NONE, HS_PREC_L1GS, HS_PREC_CHEB = 0, 1, 2
HS_BATCH_SEGMENTED, HS_BATCH_PERSISTENT = 0, 1


class HSError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"[hs status {status}] {msg}")
        self.status = status


class SingularException(HSError):
    """LinearAlgebra.SingularException(col): col is 1-based, as in Julia."""

    def __init__(self, status, msg, col):
        super().__init__(status, msg)
        self.col = col


class hs_sparse(C.Structure):
    _fields_ = [("n", C.c_int32), ("nnz", C.c_int64), ("format", C.c_int32), ("dtype", C.c_int32),
                ("ptr", C.c_void_p), ("idx", C.c_void_p), ("val", C.c_void_p)]


class hs_l1gs_info(C.Structure):
    _fields_ = [("n", C.c_int32), ("partsize", C.c_int32), ("nparts", C.c_int32), ("nchunks", C.c_int32),
                ("chunksize", C.c_int32), ("sweep", C.c_int32), ("cache", C.c_int32), ("is_sym", C.c_int32),
                ("format", C.c_int32), ("matrix_dtype", C.c_int32), ("smoother_dtype", C.c_int32),
                ("packed_len", C.c_int64), ("device_bytes", C.c_int64), ("eta", C.c_double),
                ("threads_per_part", C.c_int32), ("order", C.c_int32)]


class hs_l1gs_options(C.Structure):
    _fields_ = [("threads_per_part", C.c_int32), ("order", C.c_int32)]


class hs_cheb_info(C.Structure):
    _fields_ = [("n", C.c_int32), ("kind", C.c_int32), ("degree", C.c_int32), ("eig", C.c_int32),
                ("smoother_dtype", C.c_int32), ("rho", C.c_double), ("rho_power", C.c_double),
                ("lanczos_min", C.c_double), ("lanczos_max", C.c_double), ("astar", C.c_double)]


class hs_solve_info(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("relres", C.c_double), ("ms", C.c_double),
                ("rnorm", C.c_double)]


class hs_batch_config(C.Structure):
    _fields_ = [("max_slots", C.c_int32), ("hbm_budget", C.c_int64), ("partsize", C.c_int32), ("rtol", C.c_double),
                ("maxit", C.c_int32), ("schedule", C.c_int32)]


class hs_batch_result(C.Structure):
    _fields_ = [("tag", C.c_int64), ("iterations", C.c_int32), ("converged", C.c_int32), ("relres", C.c_double)]


class hs_batch_info(C.Structure):
    _fields_ = [("active", C.c_int32), ("finished", C.c_int32), ("hbm_used", C.c_int64), ("hbm_budget", C.c_int64),
                ("iterations_run", C.c_int64)]


_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_d = C.c_double

# name -> (restype, argtypes); every symbol of include/hsb200.h
PROTOTYPES = {
    "hs_l1gs_create": (C.c_int, [C.POINTER(hs_sparse), _i32, _i32, _d, _i32, _i32, _i32, _i32, _i32, _vp,
                                 C.POINTER(_vp)]),
    "hs_l1gs_apply": (C.c_int, [_vp, _vp, _vp, _i32, _vp]),
    "hs_l1gs_apply_host": (C.c_int, [_vp, _vp, _vp, _i32, _vp]),
    "hs_l1gs_create_opts": (C.c_int, [C.POINTER(hs_sparse), _i32, _i32, _d, _i32, _i32, _i32, _i32, _i32,
                                      C.POINTER(hs_l1gs_options), _vp, C.POINTER(_vp)]),
    "hs_l1gs_info_get": (C.c_int, [_vp, C.POINTER(hs_l1gs_info)]),
    "hs_l1gs_get_diag": (C.c_int, [_vp, _vp]),
    "hs_l1gs_get_packed": (C.c_int, [_vp, _i32, _vp, _i64]),
    "hs_l1gs_get_diag_indices": (C.c_int, [_vp, _vp]),
    "hs_l1gs_destroy": (C.c_int, [_vp]),
    "hs_matrix_create": (C.c_int, [C.POINTER(hs_sparse), _i32, _vp, C.POINTER(_vp)]),
    "hs_matrix_spmv": (C.c_int, [_vp, _vp, _vp, _d, _d, _vp]),
    "hs_matrix_destroy": (C.c_int, [_vp]),
    "hs_cheb_create": (C.c_int, [C.POINTER(hs_sparse), _i32, _i32, _i32, _i32, _vp, C.POINTER(_vp)]),
    "hs_cheb_smooth": (C.c_int, [_vp, _vp, _vp, _vp]),
    "hs_cheb_apply": (C.c_int, [_vp, _vp, _vp, _i32, _vp]),
    "hs_cheb_info_get": (C.c_int, [_vp, C.POINTER(hs_cheb_info)]),
    "hs_cheb_set_rho": (C.c_int, [_vp, _d]),
    "hs_cheb_destroy": (C.c_int, [_vp]),
    "hs_cheb_smooth_noalloc": (C.c_int, [_i32, _i64, _vp, _vp, _vp, _vp, _i32, _i32, _d, _d, _vp, _vp, _vp]),
    "hs_richardson_create": (C.c_int, [_vp, _vp, C.POINTER(_vp)]),
    "hs_richardson_smooth": (C.c_int, [_vp, _vp, _vp, _i32, _vp]),
    "hs_richardson_destroy": (C.c_int, [_vp]),
    "hs_pcg_solve": (C.c_int, [_vp, _i32, _vp, _vp, _vp, _d, _i32, _vp, C.POINTER(hs_solve_info)]),
    "hs_gmres_solve": (C.c_int, [_vp, _i32, _vp, _i32, _vp, _vp, _d, _i32, _vp, C.POINTER(hs_solve_info)]),
    "hs_cg_krylovjl": (C.c_int, [_vp, _i32, _vp, _vp, _vp, _d, _d, _i32, _vp, C.POINTER(hs_solve_info)]),
    "hs_gmres_krylovjl": (C.c_int, [_vp, _i32, _vp, _i32, _vp, _vp, _d, _d, _i32, _vp, C.POINTER(hs_solve_info)]),
    "hs_batch_create": (C.c_int, [C.POINTER(hs_batch_config), _vp, C.POINTER(_vp)]),
    "hs_batch_submit": (C.c_int, [_vp, C.POINTER(hs_sparse), _vp, _vp, _i64, _i32, C.POINTER(_i32)]),
    "hs_batch_step": (C.c_int, [_vp, _i32, C.POINTER(_i32)]),
    "hs_batch_launch": (C.c_int, [_vp, _i32]),
    "hs_batch_wait": (C.c_int, [_vp, C.POINTER(_i32)]),
    "hs_batch_poll": (C.c_int, [_vp, C.POINTER(hs_batch_result), _i32, C.POINTER(_i32)]),
    "hs_batch_info_get": (C.c_int, [_vp, C.POINTER(hs_batch_info)]),
    "hs_batch_destroy": (C.c_int, [_vp]),
    "hs_last_error": (C.c_char_p, []),
    "hs_last_singular_col": (C.c_int32, []),
    "hs_device_error": (C.c_int, [_vp, C.POINTER(_i32)]),
    "hs_kernel_launches": (C.c_int64, []),
    "hs_version": (C.c_char_p, []),
}

_lib = None


def lib():
    """Load libhsb200.so once; raise loudly if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libhsb200.so is not built ({LIB_PATH}); run __graft_entry__.build() or "
                              "make -C hybridsmoothers.jl_b200/csrc")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status == HS_OK:
        return
    L = lib()
    msg = L.hs_last_error().decode(errors="replace")
    if status == HS_ERR_SINGULAR:
        raise SingularException(status, msg, int(L.hs_last_singular_col()))
    if status == HS_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if status == HS_ERR_ARG:
        raise ValueError(msg)
    raise HSError(status, msg)


def kernel_launches():
    return int(lib().hs_kernel_launches())
