"""ctypes binding of libsvdb200.so (include/svdb200.h).

The library is the product: it is loaded from the package tree
(single-svdlib_b200/lib/libsvdb200.so) and there is no fallback.  If it is
missing, or no CUDA device is visible when a matrix is created, the call fails
with an error naming the cause.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_ROOT, "lib", "libsvdb200.so")

_lib = None
_lock = threading.Lock()

SVDB_OK = 0
STATUS_NAMES = {
    1: "ImtqlbError", 2: "StartvError", 3: "StponeError", 4: "Imtql2Error", 5: "Las2Error",
    6: "ShapeError", 7: "CudaError", 8: "TimeoutError", 9: "Unsupported", 10: "ArgumentError",
    11: "OutOfMemory", 12: "NoConvergence",
}
PRECISION = {"f64": 0, "mixed": 1}
ALGORITHM = {"lanczos": 0, "legacy": 1}
NORMALIZER = {"QR": 0, "LU": 1, "None": 2}
ORIGIN_LANCZOS, ORIGIN_LEGACY, ORIGIN_RANDOMIZED = 0, 1, 2


class svdb_diagnostics(C.Structure):
    _fields_ = [("non_zero", C.c_uint64), ("dimensions", C.c_uint64), ("iterations", C.c_uint64),
                ("transposed", C.c_int32), ("lanczos_steps", C.c_uint64),
                ("ritz_values_stabilized", C.c_uint64), ("significant_values", C.c_uint64),
                ("singular_values", C.c_uint64), ("end_interval", C.c_double * 2), ("kappa", C.c_double),
                ("random_seed", C.c_uint32)]


class svdb_rec(C.Structure):
    _fields_ = [("d", C.c_uint64), ("u_rows", C.c_uint64), ("u_cols", C.c_uint64),
                ("u", C.POINTER(C.c_double)), ("s", C.POINTER(C.c_double)),
                ("vt_rows", C.c_uint64), ("vt_cols", C.c_uint64), ("vt", C.POINTER(C.c_double)),
                ("diagnostics", svdb_diagnostics), ("on_device", C.c_int32), ("origin", C.c_int32),
                ("time_ms_total", C.c_double), ("time_ms_spmv", C.c_double), ("time_ms_ortho", C.c_double),
                ("time_ms_tridiag", C.c_double), ("time_ms_ritvec", C.c_double)]


class svdb_rec_f32(C.Structure):
    _fields_ = [("d", C.c_uint64), ("u_rows", C.c_uint64), ("u_cols", C.c_uint64),
                ("u", C.POINTER(C.c_float)), ("s", C.POINTER(C.c_float)),
                ("vt_rows", C.c_uint64), ("vt_cols", C.c_uint64), ("vt", C.POINTER(C.c_float)),
                ("diagnostics", svdb_diagnostics), ("on_device", C.c_int32), ("origin", C.c_int32),
                ("time_ms_total", C.c_double), ("time_ms_spmv", C.c_double), ("time_ms_ortho", C.c_double),
                ("time_ms_tridiag", C.c_double), ("time_ms_ritvec", C.c_double)]


class svdb_trace(C.Structure):
    _fields_ = [("alf", C.POINTER(C.c_double)), ("bet", C.POINTER(C.c_double)), ("ritz", C.POINTER(C.c_double)),
                ("bnd", C.POINTER(C.c_double)), ("cap", C.c_uint64), ("steps", C.c_uint64),
                ("purges", C.c_uint64), ("sparsity_branch", C.c_int32), ("lanczos_blocks", C.c_int32)]


class svdb_options(C.Structure):
    _fields_ = [("precision", C.c_int32), ("algorithm", C.c_int32), ("result_on_device", C.c_int32),
                ("verbose", C.c_int32), ("omega", C.POINTER(C.c_double)), ("stream", C.c_void_p),
                ("trace", C.POINTER(svdb_trace))]


class svdb_adjoint_options(C.Structure):
    _fields_ = [("precision", C.c_int32), ("inputs_on_device", C.c_int32), ("cg_tol", C.c_double),
                ("cg_max_iters", C.c_uint64), ("stream", C.c_void_p), ("cg_iterations", C.c_uint64),
                ("cg_residual", C.c_double), ("time_ms_solve", C.c_double), ("time_ms_sddmm", C.c_double)]


class svdb_batch_options(C.Structure):
    _fields_ = [("precision", C.c_int32), ("result_on_device", C.c_int32), ("autotune", C.c_int32),
                ("use_graph", C.c_int32), ("stream", C.c_void_p)]


class svdb_batch_info(C.Structure):
    _fields_ = [("count", C.c_uint64), ("subsets_per_row_item", C.c_int32), ("columns_per_lane", C.c_int32),
                ("graph_nodes", C.c_uint64), ("kernels_per_run", C.c_uint64), ("time_ms_tune", C.c_double),
                ("time_ms_last_run", C.c_double), ("total_subset_nnz", C.c_uint64)]


# Every exported symbol with its prototype: (restype, argtypes).
P = C.POINTER
u64, i64, u32, i32, dbl, vp = C.c_uint64, C.c_int64, C.c_uint32, C.c_int32, C.c_double, C.c_void_p
SIGNATURES = {
    "svdb_options_default": (None, [P(svdb_options)]),
    "svdb_matrix_create_csr": (C.c_int, [u64, u64, u64, vp, vp, vp, P(vp)]),
    "svdb_matrix_create_csc": (C.c_int, [u64, u64, u64, vp, vp, vp, P(vp)]),
    "svdb_matrix_create_coo": (C.c_int, [u64, u64, u64, vp, vp, vp, P(vp)]),
    "svdb_matrix_create_csr_device": (C.c_int, [u64, u64, u64, vp, vp, vp, P(vp)]),
    "svdb_matrix_create_csr_f32": (C.c_int, [u64, u64, u64, vp, vp, vp, P(vp)]),
    "svdb_matrix_create_csc_f32": (C.c_int, [u64, u64, u64, vp, vp, vp, P(vp)]),
    "svdb_matrix_create_coo_f32": (C.c_int, [u64, u64, u64, vp, vp, vp, P(vp)]),
    "svdb_matrix_destroy": (None, [vp]),
    "svdb_matrix_nrows": (u64, [vp]),
    "svdb_matrix_ncols": (u64, [vp]),
    "svdb_matrix_nnz": (u64, [vp]),
    "svdb_masked_new": (C.c_int, [vp, vp, u64, P(vp)]),
    "svdb_masked_with_columns": (C.c_int, [vp, vp, u64, P(vp)]),
    "svdb_masked_maps": (C.c_int, [vp, vp, vp]),
    "svdb_masked_uses_all_columns": (C.c_int, [vp]),
    "svdb_opa": (C.c_int, [vp, vp, vp, C.c_int]),
    "svdb_opb": (C.c_int, [vp, vp, vp, C.c_int]),
    "svdb_multiply_with_dense": (C.c_int, [vp, vp, u64, vp, C.c_int]),
    "svdb_multiply_transposed_by_dense": (C.c_int, [vp, vp, u64, vp]),
    "svdb_column_means": (C.c_int, [vp, vp]),
    "svdb_multiply_with_dense_centered": (C.c_int, [vp, vp, u64, vp, vp, C.c_int]),
    "svdb_multiply_transposed_by_dense_centered": (C.c_int, [vp, vp, u64, vp, vp]),
    "svdb_multiply_with_dense_device": (C.c_int, [vp, vp, u64, vp, C.c_int, C.c_int, vp]),
    "svdb_opa_device": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, vp]),
    "svdb_release_cached_memory": (C.c_int, []),
    "svdb_gram_device": (C.c_int, [vp, u64, u64, vp, C.c_int, vp]),
    "svdb_kernel_launches": (u64, []),
    "svdb_wait_selftest": (C.c_int, [C.c_int, u64]),
    "svdb_dense_split_info": (C.c_int, [vp, P(u64), P(u64)]),
    "svdb_sliced_spmv_info": (C.c_int, [vp, C.c_int, P(i32), P(i32)]),
    "svdb_tridiag_device": (C.c_int, [C.c_int, u64, vp, vp, vp, vp, vp, vp, u64, P(u64), vp, u64, P(C.c_int),
                                      P(dbl)]),
    "svdb_opb_device_noalloc": (C.c_int, [vp, vp, vp, C.c_int, vp]),
    "svdb_las2": (C.c_int, [vp, u64, u64, P(dbl), dbl, u32, P(svdb_options), P(svdb_rec)]),
    "svdb_svd": (C.c_int, [vp, P(svdb_rec)]),
    "svdb_svd_dim": (C.c_int, [vp, u64, P(svdb_rec)]),
    "svdb_svd_dim_seed": (C.c_int, [vp, u64, u32, P(svdb_rec)]),
    "svdb_legacy_svd_las2": (C.c_int, [vp, u64, u64, P(dbl), dbl, u32, P(svdb_options), P(svdb_rec)]),
    "svdb_start_vector": (C.c_int, [u32, vp, u64]),
    "svdb_las2_plan": (C.c_int, [u64, u64, u64, u64, u64, P(u64), P(u64), P(i32), P(i32)]),
    "svdb_randomized_svd": (C.c_int, [vp, u64, u64, u64, C.c_int, C.c_int, C.c_int, u64, C.c_int,
                                      P(svdb_options), P(svdb_rec)]),
    "svdb_las2_f32": (C.c_int, [vp, u64, u64, P(C.c_float), C.c_float, u32, P(svdb_options), P(svdb_rec_f32)]),
    "svdb_svd_f32": (C.c_int, [vp, P(svdb_rec_f32)]),
    "svdb_svd_dim_f32": (C.c_int, [vp, u64, P(svdb_rec_f32)]),
    "svdb_svd_dim_seed_f32": (C.c_int, [vp, u64, u32, P(svdb_rec_f32)]),
    "svdb_randomized_svd_f32": (C.c_int, [vp, u64, u64, u64, C.c_int, C.c_int, C.c_int, u64, C.c_int,
                                          P(svdb_options), P(svdb_rec_f32)]),
    "svdb_rec_f32_free": (None, [P(svdb_rec_f32)]),
    "svdb_batch_options_default": (None, [P(svdb_batch_options)]),
    "svdb_batch_create": (C.c_int, [vp, vp, vp, u64, u64, u64, u64, C.c_int, C.c_int, u64, P(svdb_batch_options),
                                    P(vp)]),
    "svdb_batch_run": (C.c_int, [vp, vp]),
    "svdb_batch_get_info": (C.c_int, [vp, P(svdb_batch_info)]),
    "svdb_batch_destroy": (None, [vp]),
    "svdb_randomized_svd_batch": (C.c_int, [vp, vp, vp, u64, u64, u64, u64, C.c_int, C.c_int, u64,
                                            P(svdb_batch_options), vp]),
    "svdb_adjoint_options_default": (None, [P(svdb_adjoint_options)]),
    "svdb_svd_adjoint": (C.c_int, [vp, u64, vp, vp, vp, vp, vp, vp, P(svdb_adjoint_options), vp]),
    "svdb_sddmm_device": (C.c_int, [vp, vp, vp, u64, vp, C.c_int, vp]),
    "svdb_svd_flip": (C.c_int, [vp, u64, u64, vp, u64, u64, C.c_int, C.c_int]),
    "svdb_rec_free": (None, [P(svdb_rec)]),
    "svdb_rec_recompose": (C.c_int, [P(svdb_rec), vp]),
    "svdb_last_error_message": (C.c_char_p, []),
    "svdb_version": (C.c_int, []),
}


def lib():
    """Load libsvdb200.so once; raise if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"libsvdb200.so not found at {LIB_PATH}: build it with `make -C single-svdlib_b200` "
                    "(the CUDA library is required; there is no CPU implementation)")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def last_error() -> str:
    return lib().svdb_last_error_message().decode(errors="replace")
