"""ctypes declarations of the C ABI in include/b2s.h (libb2sparse.so).

The library is loaded from the package directory. There is no fallback:
if the shared object is missing or fails to load, importing raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent.parent / "libb2sparse.so"

# b2s_status
OK, NOT_CONVERGED, NAN, DIVERGED, OOM, CUDA_ERROR, TIMEOUT, INVALID_ARG, INDEX_OVERFLOW, UNSUPPORTED, \
    BREAKDOWN, BUDGET, CANCELLED, IO_ERROR = range(14)
F64, F32, BOOL = 0, 1, 2
CSR, ELLPACK, SLICED_ELLPACK, CHUNKED_ELLPACK, BIELLPACK, MULTIDIAGONAL = range(6)
HOST, DEVICE = 0, 1
ABI_VERSION = 2  # B2S_ABI_VERSION of include/b2s.h
CG, BICGSTAB, GMRES, TFQMR, BICGSTABL, JACOBI, SOR = 0, 1, 2, 3, 4, 5, 6
PRECOND_NONE, PRECOND_JACOBI, PRECOND_ILU0, PRECOND_ILUT = 0, 1, 2, 3
GMRES_CGS, GMRES_CGSR, GMRES_MGS, GMRES_MGSR = range(4)
PRECISION_PLAIN, PRECISION_MIXED = 0, 1
CSR_AUTO, CSR_SCALAR, CSR_VECTOR, CSR_ADAPTIVE = range(4)


class MatrixOpts(C.Structure):
    _fields_ = [("csr_kernel", C.c_int32), ("threads_per_row", C.c_int32), ("keep_fp32_copy", C.c_int32),
                ("slice_size", C.c_int32), ("csr_row_groups", C.c_int32), ("symmetric", C.c_int32),
                ("reserved", C.c_int32 * 2)]


class MatrixInfo(C.Structure):
    _fields_ = [("format", C.c_int32), ("dtype", C.c_int32), ("rows", C.c_int32), ("cols", C.c_int32),
                ("nnz", C.c_int64), ("storage_size", C.c_int64), ("device_bytes", C.c_int64),
                ("csr_kernel", C.c_int32), ("threads_per_row", C.c_int32), ("csr_path", C.c_int32),
                ("symmetric", C.c_int32)]


class SolveOpts(C.Structure):
    _fields_ = [("solver", C.c_int32), ("preconditioner", C.c_int32), ("convergence_residue", C.c_double),
                ("divergence_residue", C.c_double), ("max_iterations", C.c_int64), ("min_iterations", C.c_int64),
                ("gmres_variant", C.c_int32), ("gmres_restarting_min", C.c_int32),
                ("gmres_restarting_max", C.c_int32), ("gmres_restarting_step_min", C.c_int32),
                ("gmres_restarting_step_max", C.c_int32), ("bicgstab_exact_residue", C.c_int32),
                ("precision", C.c_int32), ("inner_tolerance", C.c_double), ("max_refinements", C.c_int32),
                ("check_interval", C.c_int32), ("graphs", C.c_int32), ("bicgstab_ell", C.c_int32),
                ("omega", C.c_double), ("residue_period", C.c_int32), ("ilut_p", C.c_int32),
                ("ilut_threshold", C.c_double), ("reserved", C.c_int32 * 2)]


class SolveReport(C.Structure):
    _fields_ = [("status", C.c_int32), ("converged", C.c_int32), ("iterations", C.c_int64),
                ("residue", C.c_double), ("true_residual", C.c_double), ("refinements", C.c_int64),
                ("device_ms", C.c_double)]


class ServerOpts(C.Structure):
    _fields_ = [("memory_budget", C.c_int64), ("max_inflight", C.c_int32), ("mixed_min_rows", C.c_int32),
                ("reserved", C.c_int32 * 6)]


class Request(C.Structure):
    _fields_ = [("format", C.c_int32), ("rows", C.c_int32), ("nnz", C.c_int64), ("offsets", C.c_void_p),
                ("columns", C.c_void_p), ("values", C.c_void_p), ("b", C.c_void_p), ("x", C.c_void_p),
                ("opts", SolveOpts), ("reserved", C.c_int32 * 8)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("precision", C.c_int32), ("report", SolveReport),
                ("t_submit_ns", C.c_int64), ("t_admit_ns", C.c_int64), ("t_done_ns", C.c_int64),
                ("device_bytes", C.c_int64), ("t_built_ns", C.c_int64), ("t_solved_ns", C.c_int64)]


class ServerStats(C.Structure):
    _fields_ = [("memory_budget", C.c_int64), ("reserved_bytes", C.c_int64), ("peak_reserved_bytes", C.c_int64),
                ("pending", C.c_int64), ("inflight", C.c_int64), ("peak_inflight", C.c_int64),
                ("completed", C.c_int64)]


class BatchOpts(C.Structure):
    _fields_ = [("preconditioner", C.c_int32), ("cluster_size", C.c_int32), ("convergence_residue", C.c_double),
                ("divergence_residue", C.c_double), ("max_iterations", C.c_int64), ("min_iterations", C.c_int64),
                ("reserved", C.c_int32 * 8)]


class BatchReport(C.Structure):
    _fields_ = [("solves", C.c_int64), ("converged", C.c_int64), ("total_iterations", C.c_int64),
                ("max_iterations", C.c_int64), ("max_residue", C.c_double), ("device_ms", C.c_double),
                ("cluster_size", C.c_int32), ("reserved0", C.c_int32)]


class TuneOpts(C.Structure):
    _fields_ = [("reps", C.c_int32), ("warm_l2", C.c_int32), ("max_storage_ratio", C.c_double),
                ("reserved", C.c_int32 * 4)]


class TuneResult(C.Structure):
    _fields_ = [("format", C.c_int32), ("csr_kernel", C.c_int32), ("threads_per_row", C.c_int32),
                ("slice_size", C.c_int32), ("spmv_us", C.c_double), ("candidates", C.c_int32),
                ("csr_row_groups", C.c_int32), ("reserved", C.c_int32 * 4)]


class TuneEntry(C.Structure):
    _fields_ = [("format", C.c_int32), ("csr_kernel", C.c_int32), ("threads_per_row", C.c_int32),
                ("slice_size", C.c_int32), ("skipped", C.c_int32), ("csr_row_groups", C.c_int32),
                ("storage_size", C.c_int64), ("spmv_us", C.c_double)]


class Mtx(C.Structure):
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("count", C.c_int64), ("symmetric", C.c_int32),
                ("reserved", C.c_int32), ("row_indexes", C.POINTER(C.c_int32)),
                ("column_indexes", C.POINTER(C.c_int32)), ("values", C.POINTER(C.c_double))]


DUP_SET, DUP_ADD = 0, 1

_vp = C.c_void_p
_st = C.c_int

# name -> (restype, argtypes)
PROTOTYPES = {
    "b2s_status_string": (C.c_char_p, [C.c_int]),
    "b2s_last_error": (C.c_char_p, []),
    "b2s_abi_version": (C.c_int, []),
    "b2s_matrix_opts_default": (None, [C.POINTER(MatrixOpts)]),
    "b2s_matrix_create": (_st, [C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int64, _vp, _vp, _vp, C.c_int, C.c_int,
                                C.POINTER(MatrixOpts), _vp, C.POINTER(_vp)]),
    "b2s_matrix_convert": (_st, [_vp, C.c_int, C.c_int, C.POINTER(MatrixOpts), _vp, C.POINTER(_vp)]),
    "b2s_matrix_destroy": (_st, [_vp]),
    "b2s_precond_create": (_st, [_vp, C.c_int32, _vp, C.POINTER(_vp)]),
    "b2s_precond_create_ilut": (_st, [_vp, C.c_int32, C.c_double, _vp, C.POINTER(_vp)]),
    "b2s_precond_solve": (_st, [_vp, _vp, _vp, C.c_int, _vp]),
    "b2s_precond_destroy": (_st, [_vp]),
    "b2s_matrix_from_coo": (_st, [C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int64, _vp, _vp, _vp, C.c_int, C.c_int,
                                  C.c_int32, _vp, C.POINTER(MatrixOpts), _vp, C.POINTER(_vp)]),
    "b2s_mtx_read": (_st, [C.c_char_p, C.POINTER(C.POINTER(Mtx))]),
    "b2s_mtx_free": (None, [C.POINTER(Mtx)]),
    "b2s_matrix_read_mtx": (_st, [C.c_char_p, C.c_int, C.c_int, C.POINTER(MatrixOpts), _vp, C.POINTER(_vp)]),
    "b2s_matrix_write_mtx": (_st, [_vp, C.c_char_p]),
    "b2s_matrix_save": (_st, [_vp, C.c_char_p]),
    "b2s_matrix_load": (_st, [C.c_char_p, C.POINTER(MatrixOpts), _vp, C.POINTER(_vp)]),
    "b2s_matrix_get_info": (_st, [_vp, C.POINTER(MatrixInfo)]),
    "b2s_matrix_export": (_st, [_vp, C.c_char_p, _vp, C.c_int64, C.POINTER(C.c_int64)]),
    "b2s_matrix_export_range": (_st, [_vp, C.c_char_p, C.c_int64, C.c_int64, _vp]),
    "b2s_spmv": (_st, [_vp, _vp, _vp, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int, _vp]),
    "b2s_spmv_ex": (_st, [_vp, _vp, _vp, C.c_int, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int, _vp]),
    "b2s_matrix_device_status": (_st, [_vp, _vp]),
    "b2s_dot": (_st, [C.c_int, C.c_int64, _vp, _vp, _vp, _vp]),
    "b2s_norm2": (_st, [C.c_int, C.c_int64, _vp, _vp, _vp]),
    "b2s_axpby": (_st, [C.c_int, C.c_int64, C.c_double, _vp, C.c_double, _vp, _vp]),
    "b2s_gather": (_st, [C.c_int32, C.c_int64, _vp, C.c_int64, _vp, _vp, _vp]),
    "b2s_scan_i32": (_st, [C.c_int64, _vp, C.c_int32, _vp]),
    "b2s_solve_opts_default": (None, [C.POINTER(SolveOpts)]),
    "b2s_solver_create": (_st, [_vp, C.POINTER(SolveOpts), C.POINTER(_vp)]),
    "b2s_solver_destroy": (_st, [_vp]),
    "b2s_solve": (_st, [_vp, _vp, _vp, C.c_int, _vp, C.POINTER(SolveReport)]),
    "b2s_scan_i32_noalloc": (_st, [C.c_int64, _vp, C.c_int32, _vp]),
    "b2s_matrix_permute_rows": (_st, [_vp, _vp, C.c_int, _vp]),
    "b2s_matrix_permute_columns": (_st, [_vp, _vp, C.c_int, _vp]),
    "b2s_matrix_reorder": (_st, [_vp, _vp, _vp, C.c_int, _vp, C.POINTER(_vp)]),
    "b2s_reorder_array": (_st, [C.c_int32, C.c_int64, _vp, _vp, _vp, _vp]),
    "b2s_tune_opts_default": (None, [C.POINTER(TuneOpts)]),
    "b2s_autotune_spmv": (_st, [_vp, C.c_int, C.POINTER(TuneOpts), _vp, C.POINTER(TuneResult), _vp, C.c_int32,
                                C.POINTER(C.c_int32)]),
    "b2s_batch_opts_default": (None, [C.POINTER(BatchOpts)]),
    "b2s_batch_create": (_st, [C.c_int32, _vp, _vp, _vp, _vp, _vp, C.c_int, C.POINTER(BatchOpts), _vp,
                               C.POINTER(_vp)]),
    "b2s_batch_solve": (_st, [_vp, _vp, _vp, _vp, C.POINTER(BatchReport)]),
    "b2s_batch_results": (_st, [_vp, _vp, _vp, _vp]),
    "b2s_batch_destroy": (_st, [_vp]),
    "b2s_server_opts_default": (None, [C.POINTER(ServerOpts)]),
    "b2s_server_clock_ns": (C.c_int64, []),
    "b2s_server_create": (_st, [C.POINTER(ServerOpts), C.POINTER(_vp)]),
    "b2s_server_submit": (_st, [_vp, C.POINTER(Request), C.POINTER(C.c_int64)]),
    "b2s_server_wait": (_st, [_vp, C.c_int64, C.c_double, C.POINTER(RequestResult)]),
    "b2s_server_get_stats": (_st, [_vp, C.POINTER(ServerStats)]),
    "b2s_server_destroy": (_st, [_vp]),
}


def load(path: Path = LIB_PATH) -> C.CDLL:
    if not path.exists():
        raise ImportError(f"{path} is not built: run __graft_entry__.build() (nvcc, sm_100a)")
    lib = C.CDLL(str(path))
    for name, (res, args) in PROTOTYPES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if lib.b2s_abi_version() != ABI_VERSION:
        raise ImportError(f"{path} has ABI {lib.b2s_abi_version()}, these bindings ABI {ABI_VERSION}: rebuild it")
    return lib
