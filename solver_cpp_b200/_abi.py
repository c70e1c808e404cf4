"""ctypes declarations of the C ABI in include/krylov_sm100.h.

The shared library is built in-tree (``make -C solver_cpp_b200/csrc``) and
loaded from this package directory. There is no fallback: if the library is
missing, importing the compute API raises.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libkrylov_sm100.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)

# ks_status
KS_OK = 0
KS_NOT_CONVERGED = 2
KS_BREAKDOWN = 3
KS_NAN_DETECTED = 4
KS_BAD_INPUT = 5
KS_CUDA_ERROR = 6
KS_TIMEOUT = 7
KS_OUT_OF_MEMORY = 8
KS_NO_DEVICE = 9
KS_IO_ERROR = 10
KS_UNIMPLEMENTED = 99

# ks_solver (values of the reference's SOLVERS_NAME)
SOLVERS = {
    "NONE": 0, "CG": 1, "BICG": 2, "CR": 3, "GCR": 4, "GMRES": 5,
    "KSKIPCG": 6, "KSKIPCR": 7, "KSKIPBICG": 8, "VPCG": 9, "VPBICG": 10,
    "VPCR": 11, "VPGCR": 12, "VPGMRES": 13,
}

# ks_precision
FP64, FP32, BF16 = 0, 1, 2
PRECISIONS = {"fp64": FP64, "fp32": FP32, "bf16": BF16}

MAT_TRANSPOSE = 1
MAT_FP32 = 2
MAT_BF16 = 4
MAT_INDEX32 = 8
MAT_NO_DIAG = 16


ABI_VERSION = 4  # KS_ABI_VERSION of the header these structures mirror


class Params(C.Structure):
    _fields_ = [
        ("outer_maxloop", C.c_int64), ("outer_eps", C.c_double), ("outer_restart", C.c_int64),
        ("outer_kskip", C.c_int32), ("outer_fix", C.c_int32),
        ("inner_maxloop", C.c_int64), ("inner_eps", C.c_double), ("inner_restart", C.c_int64),
        ("inner_kskip", C.c_int32), ("inner_fix", C.c_int32),
        ("inner_precision", C.c_int32), ("reference_defects", C.c_int32),
        ("transpose", C.c_int32), ("poll_interval", C.c_int32), ("x_update", C.c_int32),
        ("cluster_solve", C.c_int32), ("inner_fast", C.c_int32), ("true_residual", C.c_int32),
        ("profile", C.c_int32), ("reserved0", C.c_int32), ("x_ref", C.c_void_p),
    ]


class Report(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("loop", C.c_int64), ("hist_len", C.c_int64),
        ("final_rel_res", C.c_double), ("true_res_log10", C.c_double), ("true_rel_res", C.c_double),
        ("spmv_count", C.c_int64), ("inner_iterations", C.c_int64), ("solve_seconds", C.c_double),
        ("x_rel_diff", C.c_double), ("true_residual_checks", C.c_int64),
        ("t_mv", C.c_double), ("t_dot", C.c_double), ("t_other", C.c_double), ("t_memset", C.c_double),
        ("t_h2d", C.c_double), ("t_d2h", C.c_double),
        ("n_mv", C.c_int64), ("n_dot", C.c_int64), ("n_other", C.c_int64), ("n_memset", C.c_int64),
        ("t_mv_low", C.c_double), ("n_mv_low", C.c_int64),
    ]


# (name, restype, argtypes). Every symbol the header declares.
_VP = C.c_void_p
_I64 = C.c_int64
_D = C.c_double
_PD = C.POINTER(C.c_double)
_PI64 = C.POINTER(C.c_int64)
_PI32 = C.POINTER(C.c_int32)
SIGNATURES = [
    ("ks_ctx_create", C.c_int, [C.c_int, C.POINTER(_VP)]),
    ("ks_ctx_destroy", C.c_int, [_VP]),
    ("ks_ctx_set_stream", C.c_int, [_VP, _VP]),
    ("ks_ctx_synchronize", C.c_int, [_VP]),
    ("ks_device_count", C.c_int, []),
    ("ks_status_string", C.c_char_p, [C.c_int]),
    ("ks_ctx_launches", C.c_int64, [_VP]),
    ("ks_last_error", C.c_char_p, [_VP]),
    ("ks_abi_version", C.c_int, []),
    ("ks_ctx_set_wait_limit", C.c_int, [_VP, C.c_int64]),
    ("ks_csr_upload", C.c_int, [_VP, _I64, _I64, _VP, _VP, _VP, C.c_uint, C.POINTER(_VP)]),
    ("ks_csr_upload_device", C.c_int, [_VP, _I64, _I64, _VP, _VP, _VP, C.c_uint, C.POINTER(_VP)]),
    ("ks_mat_destroy", C.c_int, [_VP]),
    ("ks_mat_info", C.c_int, [_VP, _PI64, _PI64, _PI64]),
    ("ks_mat_index_bytes", C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("ks_mat_diagonals", C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("ks_mat_dia_symmetric", C.c_int, [_VP, _PI32, _PI32]),
    ("ks_mat_transpose_download", C.c_int, [_VP, _VP, _VP, _VP]),
    ("ks_vec_create", C.c_int, [_VP, _I64, C.c_int, C.POINTER(_VP)]),
    ("ks_vec_wrap", C.c_int, [_VP, _I64, C.c_int, _VP, C.POINTER(_VP)]),
    ("ks_vec_destroy", C.c_int, [_VP]),
    ("ks_vec_upload", C.c_int, [_VP, _VP]),
    ("ks_vec_download", C.c_int, [_VP, _VP]),
    ("ks_vec_upload_range", C.c_int, [_VP, _I64, _I64, _VP]),
    ("ks_vec_download_range", C.c_int, [_VP, _I64, _I64, _VP]),
    ("ks_vec_fill", C.c_int, [_VP, _D]),
    ("ks_vec_device_ptr", _VP, [_VP]),
    ("ks_vec_length", _I64, [_VP]),
    ("ks_spmv", C.c_int, [_VP, C.c_int, _VP, _VP]),
    ("ks_spmv_values", C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP]),
    ("ks_dot", C.c_int, [_VP, _VP, _PD]),
    ("ks_nrm2", C.c_int, [_VP, _PD]),
    ("ks_axpy", C.c_int, [_D, _VP, _VP]),
    ("ks_axpy_dot", C.c_int, [_D, _VP, _VP, _VP, _PD]),
    ("ks_block_dot", C.c_int, [_VP, _I64, C.c_int, _VP, _VP]),
    ("ks_block_dot_noalloc", C.c_int, [_VP, _I64, C.c_int, _VP, _I64, _VP, _VP]),
    ("ks_block_axpy", C.c_int, [_VP, _I64, C.c_int, _VP, _VP]),
    ("ks_matpow", C.c_int, [_VP, _VP, _VP, C.c_int, _VP, _VP]),
    ("ks_gram_cg", C.c_int, [_VP, _VP, _VP, _VP, C.c_int, _VP, _VP, _VP]),
    ("ks_gram_bicg", C.c_int, [_VP, _VP, _VP, _VP, C.c_int, _VP, _VP, _VP, _VP]),
    ("ks_params_default", None, [C.POINTER(Params)]),
    ("ks_solve", C.c_int, [_VP, _VP, C.c_int, C.c_int, C.POINTER(Params), _VP, _VP, _VP, _VP, _I64,
                           C.POINTER(Report)]),
    ("ks_solve_host", C.c_int, [_VP, _VP, C.c_int, C.c_int, C.POINTER(Params), _VP, _VP, _VP, _VP, _I64,
                                C.POINTER(Report)]),
    ("ks_check_error", C.c_int, [_VP, _VP, _VP, _PD, _PD]),
    ("ks_adjoint_grad", C.c_int, [_VP, _VP, C.c_int, C.c_int, C.POINTER(Params), _VP, _VP, _VP, _VP,
                                  C.POINTER(Report)]),
    ("ks_pattern_grad", C.c_int, [_VP, _VP, _VP, _VP]),
    ("ks_crs_read_header", C.c_int, [C.c_char_p, _PI64, _PI64]),
    ("ks_crs_read", C.c_int, [C.c_char_p, _I64, _I64, _VP, _VP, _VP, _VP, _VP]),
    ("ks_partition_rows", C.c_int, [_I64, C.c_int, _I64, _VP]),
    ("ks_halo_window", C.c_int, [_I64, _I64, _VP, _VP, _PI64, _PI64]),
    ("ks_halo_plan", C.c_int, [C.c_int, C.c_int, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    ("ks_comm_unique_id", C.c_int, [_VP]),
    ("ks_comm_create_nccl", C.c_int, [_VP, C.c_int, C.c_int, _VP, C.POINTER(_VP)]),
    ("ks_comm_create_local", C.c_int, [_VP, C.c_int, _VP]),
    ("ks_comm_destroy", C.c_int, [_VP]),
    ("ks_comm_info", C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("ks_dist_upload", C.c_int, [_VP, _VP, _I64, _I64, _I64, _VP, _VP, _VP, _VP, _VP, _VP, C.c_uint, C.POINTER(_VP)]),
    ("ks_mat_dist_info", C.c_int, [_VP, _PI64, _PI64, _PI64, _PI64, _PI64]),
    ("ks_mm_read_header", C.c_int, [C.c_char_p, _PI64, _PI64]),
    ("ks_mm_read", C.c_int, [C.c_char_p, _I64, _I64, _VP, _VP, _VP]),
    ("ks_crs_write", C.c_int, [C.c_char_p, _I64, _I64, _VP, _VP, _VP, _VP, _VP]),
]

_lib = None


class LibraryMissing(RuntimeError):
    pass


def load():
    """Load the in-tree CUDA library (raises LibraryMissing if absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LibraryMissing(
            f"{LIB_NAME} not found in {PKG_DIR}; build it with `make -C solver_cpp_b200/csrc` "
            "(or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.ks_abi_version() != ABI_VERSION:  # the structures above would not match
        raise LibraryMissing(f"{LIB_NAME} has ABI version {lib.ks_abi_version()}, the binding expects "
                             f"{ABI_VERSION}; rebuild it with `make -C solver_cpp_b200/csrc`")
    _lib = lib
    return lib
