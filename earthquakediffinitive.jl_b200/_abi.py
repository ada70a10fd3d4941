"""ctypes binding of libeqd (include/eqd.h).

The library must be built (build.py). Loading fails loudly when it is
missing; there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# EQD_LIB selects another build of the library (e.g. a debug build).
LIB_PATH = os.environ.get("EQD_LIB") or os.path.join(HERE, "lib", "libeqd.so")

EQD_OK = 0
EQD_ERR_ARG = 1
EQD_ERR_OOM = 2
EQD_ERR_CUDA = 3
EQD_ERR_NOT_CONVERGED = 4
EQD_ERR_TIMEOUT = 5
EQD_ERR_UNSUPPORTED = 6
EQD_ERR_NO_DEVICE = 7

EQD_PREC_FP64 = 0
EQD_PREC_MIXED = 1
EQD_PRECOND_NONE = 0
EQD_PRECOND_JACOBI = 1
EQD_FLAG_STRICT = 1
EQD_FLAG_NO_SPLIT = 2
EQD_FLAG_FUSE = 4

COL_CONVERGED = 1
COL_MAXITER = 2
COL_BREAKDOWN = 3
COL_NONFINITE = 4


class GridDesc(C.Structure):
    _fields_ = [("n1", C.c_int32), ("n2", C.c_int32), ("n3", C.c_int32),
                ("x1_extent", C.c_double),
                ("x2_lo", C.c_double), ("x2_hi", C.c_double),
                ("x3_lo", C.c_double), ("x3_hi", C.c_double),
                ("lam", C.c_double), ("mu", C.c_double), ("l_f", C.c_double),
                ("order", C.c_int32), ("device", C.c_int32)]


class SolveOpts(C.Structure):
    _fields_ = [("rtol", C.c_double), ("atol", C.c_double), ("itmax", C.c_int64),
                ("precond", C.c_int32), ("precision", C.c_int32), ("chunk", C.c_int32),
                ("reliable_delta", C.c_double), ("hbm_budget_bytes", C.c_uint64),
                ("variant", C.c_int32), ("flags", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("solves", C.c_int64), ("iterations", C.c_int64),
                ("max_iterations", C.c_int64), ("unconverged", C.c_int64),
                ("reliable_updates", C.c_int64), ("seconds", C.c_double),
                ("device_seconds", C.c_double), ("precond", C.c_int32),
                ("precision", C.c_int32), ("kernel_launches", C.c_int64)]


# Every symbol include/eqd.h declares (the ABI test checks they are exported).
EXPORTS = [
    "eqd_last_error", "eqd_version", "eqd_default_opts", "eqd_device_count",
    "eqd_grid_create", "eqd_grid_destroy", "eqd_grid_info", "eqd_grid_fault_axes",
    "eqd_apply", "eqd_cg_solve", "eqd_shear_traction", "eqd_stiffness_exact",
    "eqd_stiffness_columns", "eqd_stiffness_columns_device", "eqd_stiffness_toeplitz", "eqd_diag",
    "eqd_profile_apply", "eqd_autotune", "eqd_set_variant", "eqd_test_inject_wait_timeout", "eqd_assemble",
    "eqd_tune_chunk",
    "eqd_kmat_create", "eqd_kmat_gemv", "eqd_kmat_gemv_device", "eqd_kmat_destroy", "eqd_kmat_gemv_static",
    "eqd_server_create", "eqd_server_add_grid", "eqd_server_submit", "eqd_server_wait",
    "eqd_server_poll", "eqd_server_request_info", "eqd_server_release", "eqd_server_destroy",
    "eqd_rhs_create", "eqd_rhs_eval", "eqd_rhs_fields", "eqd_rhs_report", "eqd_rhs_destroy", "eqd_friction_solve",
]


class RequestInfo(C.Structure):
    """`eqd_request_info` (include/eqd.h)."""
    _fields_ = [("state", C.c_int32), ("ncols", C.c_int32), ("unconverged", C.c_int32),
                ("max_iterations", C.c_int32), ("iterations", C.c_int64), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_done", C.c_double)]


class EqdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[eqd {code}] {msg}")
        self.code = code


class EqdArgumentError(EqdError, ValueError):
    """Misuse: the reference raises `ErrorException` via `error()` here."""


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libeqd.so is not built ({LIB_PATH}); run "
                              "`python earthquakediffinitive.jl_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        L.eqd_last_error.restype = C.c_char_p
        L.eqd_version.restype = C.c_char_p
        for name in EXPORTS:
            if name not in ("eqd_last_error", "eqd_version", "eqd_default_opts"):
                getattr(L, name).restype = C.c_int
        L.eqd_default_opts.restype = None
        _lib = L
    return _lib


def check(rc):
    if rc != EQD_OK:
        msg = lib().eqd_last_error().decode(errors="replace")
        cls = EqdArgumentError if rc == EQD_ERR_ARG else EqdError
        raise cls(rc, msg)


def ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def default_opts():
    o = SolveOpts()
    lib().eqd_default_opts(C.byref(o))
    return o
