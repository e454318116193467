"""ctypes binding of libcfdgpu.so (the C ABI declared in include/cfdgpu.h).

The shared library is built in-tree (``cfdrs_b200/libcfdgpu.so``) by
``cfdrs_b200.build.build()``. There is no CPU fallback: if the library is
missing, or no CUDA device is present, the first call raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# CFDGPU_LIB selects another build of the same library (e.g. the sanitizer build).
LIB_PATH = os.environ.get("CFDGPU_LIB") or os.path.join(_HERE, "libcfdgpu.so")

CFD_OK = 0
STATUS_NAMES = {0: "CFD_OK", 1: "CFD_ERR_DIM", 2: "CFD_ERR_CONFIG", 3: "CFD_ERR_CUDA",
                4: "CFD_ERR_TIMEOUT", 5: "CFD_ERR_NONFINITE", 6: "CFD_ERR_ALLOC", 7: "CFD_ERR_STATE"}

# Every symbol include/cfdgpu.h declares (checked by the ABI test).
EXPORTS = [
    "cfd_last_error", "cfd_version",
    "cfd_context_create", "cfd_context_set_stream", "cfd_context_synchronize", "cfd_context_destroy",
    "cfd_csr_create", "cfd_csr_create_i32", "cfd_csr_update_values", "cfd_csr_info", "cfd_csr_destroy",
    "cfd_csr_layout", "cfd_csr_set_path", "cfd_layout_check",
    "cfd_spmv", "cfd_spmv_f32",
    "cfd_amg_config_default", "cfd_amg_setup", "cfd_amg_recompute", "cfd_amg_apply", "cfd_amg_stats",
    "cfd_amg_level", "cfd_amg_set_path", "cfd_amg_destroy", "cfd_amg_setup_host", "cfd_selftest_wait_timeout",
    "cfd_saddle_setup", "cfd_simple_apply", "cfd_block_diagonal_apply", "cfd_simple_apply_host",
    "cfd_block_diagonal_host", "cfd_component_block_setup", "cfd_component_block_apply",
    "cfd_darcy2d_assemble", "cfd_darcy2d_theta_grad", "cfd_context_set_cluster_solve", "cfd_adjoint",
    "cfd_solve_options_default", "cfd_solve", "cfd_last_kernel_stats",
    "cfd_pattern_outer", "cfd_csr_set_values_device",
    "cfd_batch_create", "cfd_batch_update_values", "cfd_batch_solve", "cfd_batch_autotune", "cfd_batch_config",
    "cfd_batch_groups", "cfd_batch_set_config",
    "cfd_batch_create_networks", "cfd_batch_assemble", "cfd_batch_values", "cfd_network_assemble_host",
    "cfd_batch_destroy", "cfd_ls_options_default", "cfd_batch_linear_system_solve",
    "cfd_residual_norm_noalloc",
]


class AmgConfigC(C.Structure):
    _fields_ = [("max_levels", C.c_int32), ("coarsening", C.c_int32), ("min_coarse_size", C.c_int64),
                ("interpolation", C.c_int32), ("smoother", C.c_int32), ("pre_smooth", C.c_int32),
                ("post_smooth", C.c_int32), ("relaxation", C.c_double), ("strength_threshold", C.c_double),
                ("coarse_solve", C.c_int32), ("coarse_sweeps", C.c_int32), ("aggregate_size", C.c_int64),
                ("seed", C.c_uint64), ("coarse_order", C.c_int32), ("max_interp_points", C.c_int32)]


class AmgStatsC(C.Structure):
    _fields_ = [("num_levels", C.c_int32), ("pad", C.c_int32), ("level_rows", C.c_int64 * 16),
                ("level_nnz", C.c_int64 * 16), ("operator_complexity", C.c_double),
                ("grid_complexity", C.c_double), ("setup_seconds", C.c_double)]


class SolverConfigC(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("relative_tolerance", C.c_double), ("max_iterations", C.c_int64)]


class SolveOptionsC(C.Structure):
    _fields_ = [("solver", C.c_int32), ("precond", C.c_int32), ("precision", C.c_int32),
                ("memory", C.c_int32), ("inner_tolerance", C.c_double), ("max_outer", C.c_int32),
                ("check_every", C.c_int32), ("restart", C.c_int32)]


class SolveReportC(C.Structure):
    _fields_ = [("termination", C.c_int32), ("outer_iterations", C.c_int32), ("iterations", C.c_int64),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("threshold", C.c_double), ("device_ms", C.c_double)]


class BatchReportC(C.Structure):
    _fields_ = [("num_systems", C.c_int32), ("converged_systems", C.c_int32), ("total_iterations", C.c_int64),
                ("max_iterations", C.c_int32), ("pad", C.c_int32), ("max_rel_residual", C.c_double),
                ("device_ms", C.c_double), ("direct_ms", C.c_double), ("krylov_ms", C.c_double),
                ("fallback_ms", C.c_double)]


class LsOptionsC(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iterations", C.c_int64), ("method", C.c_int32),
                ("precision", C.c_int32), ("memory", C.c_int32), ("max_outer", C.c_int32),
                ("inner_tolerance", C.c_double)]


class LsResultC(C.Structure):
    _fields_ = [("method", C.c_int32), ("path", C.c_int32), ("termination", C.c_int32),
                ("iterations", C.c_int32), ("residual", C.c_double)]


class LayoutInfoC(C.Structure):
    _fields_ = [("blocks", C.c_int64), ("compressed_nnz", C.c_int64), ("all_compressed", C.c_int32),
                ("x_staged", C.c_int32), ("threads_per_row", C.c_int32), ("max_windows", C.c_int32),
                ("staged_x_entries", C.c_int64), ("path_f32", C.c_int32), ("path_f64", C.c_int32),
                ("sliced", C.c_int32), ("diagonals", C.c_int32), ("sliced_slots", C.c_int64)]


class KernelStatsC(C.Structure):
    _fields_ = [("launches", C.c_int64), ("spmv_launches", C.c_int64), ("spmv_bytes", C.c_double)]


class CfdError(RuntimeError):
    """A non-numerical failure of the C ABI (Rust ``Err`` in the reference)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def load():
    """Load libcfdgpu.so, raising if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -c 'import cfdrs_b200.build as b; b.build()'` "
            "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    PP = C.POINTER(C.c_void_p)
    sig = {
        "cfd_last_error": (C.c_char_p, []),
        "cfd_version": (C.c_char_p, []),
        "cfd_context_create": (C.c_int, [C.c_int, PP]),
        "cfd_context_set_stream": (C.c_int, [P, P]),
        "cfd_context_synchronize": (C.c_int, [P]),
        "cfd_context_destroy": (C.c_int, [P]),
        "cfd_csr_create": (C.c_int, [P, I64, I64, I64, P, P, P, PP]),
        "cfd_csr_create_i32": (C.c_int, [P, I64, I64, I64, P, P, P, PP]),
        "cfd_csr_update_values": (C.c_int, [P, P]),
        "cfd_csr_info": (C.c_int, [P, P, P, P]),
        "cfd_csr_destroy": (C.c_int, [P]),
        "cfd_csr_layout": (C.c_int, [P, P]),
        "cfd_csr_set_path": (C.c_int, [P, I32, I32]),
        "cfd_layout_check": (C.c_int, [I64, I64, I64, P, P, P, P, P, P]),
        "cfd_spmv": (C.c_int, [P, P, P]),
        "cfd_spmv_f32": (C.c_int, [P, P, P]),
        "cfd_amg_config_default": (None, [P]),
        "cfd_amg_setup": (C.c_int, [P, P, PP]),
        "cfd_amg_recompute": (C.c_int, [P, P]),
        "cfd_amg_apply": (C.c_int, [P, P, P]),
        "cfd_amg_stats": (C.c_int, [P, P]),
        "cfd_amg_level": (C.c_int, [P, C.c_int, C.c_int, P, P, P, P, P, P]),
        "cfd_amg_setup_host": (C.c_int, [C.c_int64, P, P, P, P, PP]),
        "cfd_selftest_wait_timeout": (C.c_int, [P, C.c_int32]),
        "cfd_amg_set_path": (C.c_int, [P, I32, I32]),
        "cfd_amg_destroy": (C.c_int, [P]),
        "cfd_solve_options_default": (None, [P]),
        "cfd_solve": (C.c_int, [P, P, P, P, P, P, P]),
        "cfd_last_kernel_stats": (C.c_int, [P, P]),
        "cfd_pattern_outer": (C.c_int, [P, P, P, D, P]),
        "cfd_csr_set_values_device": (C.c_int, [P, P]),
        "cfd_batch_create": (C.c_int, [P, I32, P, P, P, P, PP]),
        "cfd_saddle_setup": (C.c_int, [P, C.c_int64]),
        "cfd_simple_apply": (C.c_int, [P, P, P]),
        "cfd_block_diagonal_apply": (C.c_int, [P, P, P]),
        "cfd_component_block_setup": (C.c_int, [P, C.c_int64, C.c_double]),
        "cfd_component_block_apply": (C.c_int, [P, P, P]),
        "cfd_darcy2d_assemble": (C.c_int, [P, C.c_int64, P, P, P]),
        "cfd_context_set_cluster_solve": (C.c_int, [P, I32]),
        "cfd_adjoint": (C.c_int, [P, P, P, P, P, P, P, I32, P, P]),
        "cfd_darcy2d_theta_grad": (C.c_int, [P, C.c_int64, P, P, P, P]),
        "cfd_block_diagonal_host": (C.c_int, [C.c_int64, P, P, P, C.c_int64, P]),
        "cfd_simple_apply_host": (C.c_int, [C.c_int64, P, P, P, C.c_int64, P, P]),
        "cfd_batch_create_networks": (C.c_int, [P, I32, P, P, P, P, P, P, PP]),
        "cfd_batch_assemble": (C.c_int, [P, P, P, I32]),
        "cfd_batch_values": (C.c_int, [P, P, P]),
        "cfd_network_assemble_host": (C.c_int, [I32, P, P, P, P, P, P, P, P, P, P, P, P, P]),
        "cfd_batch_update_values": (C.c_int, [P, P]),
        "cfd_batch_solve": (C.c_int, [P, P, P, P, P, P, P, P, P]),
        "cfd_batch_autotune": (C.c_int, [P, I32, I32]),
        "cfd_batch_config": (C.c_int, [P, I32, P, P, P]),
        "cfd_batch_groups": (C.c_int, [P, I32, P]),
        "cfd_batch_set_config": (C.c_int, [P, I32, P, P]),
        "cfd_batch_destroy": (C.c_int, [P]),
        "cfd_ls_options_default": (None, [P]),
        "cfd_batch_linear_system_solve": (C.c_int, [P, P, P, P, P, P]),
        "cfd_residual_norm_noalloc": (C.c_int, [I64, I64, P, P, P, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != CFD_OK:
        msg = load().cfd_last_error()
        raise CfdError(status, msg.decode() if msg else "")
