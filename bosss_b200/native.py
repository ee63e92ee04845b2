"""ctypes binding of ``lib/libbsgpu.so`` (the C ABI declared in ``include/bsgpu.h``).

There is no fallback: if the library is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libbsgpu.so")

OK, ERR_ARGUMENT, ERR_CUDA, ERR_ARITHMETIC, ERR_NOMEM, ERR_UNSUPPORTED, ERR_TIMEOUT = range(7)
HOST_POINTERS, DEVICE_POINTERS = 0, 1
COB_EYE, COB_DIAG_BLOCK_EQUILIB = 0, 1
SOLVER_SOFTPCG, SOLVER_FGMRES_PMG, SOLVER_ORTHOMG, SOLVER_BLOCKJACOBI, SOLVER_SOFTGMRES = 0, 1, 2, 3, 4
TERM_DEFAULT, TERM_RELATIVE = 0, 1
COARSE_DENSE, COARSE_PCG, COARSE_AMG, COARSE_HMG = 0, 1, 2, 3
PRECISION_FP64, PRECISION_MIXED = 0, 1
FP16_MATRICES = 2
SMOOTHER_BLOCKJACOBI, SMOOTHER_BLOCKGS, SMOOTHER_SCHWARZ, SMOOTHER_ILU, SMOOTHER_ILU_NATURAL = 0, 1, 2, 3, 4
SMOOTHER_SCHWARZ_BLOCKS = 5
LEARNED_OFF, LEARNED_FGMRES, LEARNED_PRESMOOTH, LEARNED_BOTH = 0, 1, 2, 3

# every symbol the header declares (checked by the CPU test-suite)
EXPORTS = [
    "bsgpu_get_version", "bsgpu_last_error", "bsgpu_get_launch_count", "bsgpu_set_device",
    "bsgpu_matrix_autotune", "bsgpu_autotune_report",
    "bsgpu_matrix_create", "bsgpu_matrix_destroy", "bsgpu_matrix_get_info", "bsgpu_matrix_read_values",
    "bsgpu_matrix_spmv", "bsgpu_matrix_spmv_noalloc", "bsgpu_matrix_spmv_device", "bsgpu_matrix_create_single",
    "bsgpu_matrix_spmv_device_f32",
    "bsgpu_matrix_restrict",
    "bsgpu_mgop_create", "bsgpu_mgop_destroy", "bsgpu_mgop_get_operator", "bsgpu_mgop_add_h_level",
    "bsgpu_mgop_set_cell_neighbours", "bsgpu_mgop_set_cell_features", "bsgpu_mgop_read_left_cob",
    "bsgpu_solver_train_learned",
    "bsgpu_solver_config_default", "bsgpu_solver_create", "bsgpu_solver_destroy", "bsgpu_solver_solve",
    "bsgpu_solver_solve_device", "bsgpu_solver_get_history", "bsgpu_solver_set_tracing", "bsgpu_solver_get_trace",
    "bsgpu_solver_learned_info", "bsgpu_solver_learned_get_weights", "bsgpu_solver_learned_set_weights",
    "bsgpu_solver_learned_apply", "bsgpu_solver_learned_gradient",
    "bsgpu_batch_create", "bsgpu_batch_solve_device", "bsgpu_batch_destroy", "bsgpu_assemble_sip_cartesian",
    "bsgpu_sip_templates", "bsgpu_schwarz_blocks", "bsgpu_ilu_wavefronts", "bsgpu_project_separable",
]


class SolverConfig(C.Structure):
    _fields_ = [("solver", C.c_int32), ("termination", C.c_int32), ("tol", C.c_double), ("max_iter", C.c_int32),
                ("min_iter", C.c_int32), ("max_krylov", C.c_int32), ("n_levels", C.c_int32),
                ("level_keep", C.c_int32 * 8), ("post_sweeps", C.c_int32), ("bj_iters", C.c_int32),
                ("bj_omega", C.c_double), ("coarse_kind", C.c_int32), ("coarse_tol", C.c_double),
                ("coarse_max_iter", C.c_int32), ("sub_max_iter", C.c_int32), ("sub_reduction", C.c_double),
                ("precision", C.c_int32), ("h_levels", C.c_int32), ("h_sweeps", C.c_int32), ("h_cycle", C.c_int32),
                ("dense_limit", C.c_int32), ("smoother", C.c_int32), ("h_smoother", C.c_int32),
                ("learned", C.c_int32), ("learned_hidden", C.c_int32), ("learned_stall", C.c_double),
                ("ortho_max_krylov", C.c_int32), ("recalc_resi_period", C.c_int32), ("learned_pairs", C.c_int32),
                ("graph", C.c_int32), ("autotune", C.c_int32), ("fp16_storage", C.c_int32),
                ("schwarz_parts", C.c_int32), ("schwarz_overlap", C.c_int32), ("schwarz_scaling", C.c_int32),
                ("reserved", C.c_int32 * 5)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("nested", C.c_int32), ("converged", C.c_int32),
                ("n_history", C.c_int32), ("res0", C.c_double), ("res", C.c_double), ("seconds", C.c_double)]


class BsgpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"bsgpu error {code}: {msg}")
        self.code = code


class BsgpuArgumentError(BsgpuError, ValueError):
    pass


class BsgpuArithmeticError(BsgpuError, ArithmeticError):
    pass


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m bosss_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, dbl, flt = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_float
        sig = {
            "bsgpu_get_version": [vp, vp],
            "bsgpu_last_error": [C.c_char_p, C.c_size_t],
            "bsgpu_get_launch_count": [vp],
            "bsgpu_set_device": [C.c_int],
            "bsgpu_matrix_autotune": [vp],
            "bsgpu_autotune_report": [C.c_char_p, C.c_size_t],
            "bsgpu_matrix_create": [vp, i64, i32, vp, vp, vp, vp, i32],
            "bsgpu_matrix_destroy": [vp],
            "bsgpu_matrix_get_info": [vp, vp, vp, vp, vp],
            "bsgpu_matrix_read_values": [vp, vp, i32],
            "bsgpu_matrix_spmv": [vp, dbl, vp, dbl, vp],
            "bsgpu_matrix_spmv_noalloc": [vp, dbl, vp, dbl, vp],
            "bsgpu_matrix_spmv_device": [vp, dbl, vp, dbl, vp, vp],
            "bsgpu_matrix_create_single": [vp, vp],
            "bsgpu_matrix_spmv_device_f32": [vp, flt, vp, flt, vp, vp],
            "bsgpu_matrix_restrict": [vp, i32, vp],
            "bsgpu_mgop_create": [vp, vp, i32],
            "bsgpu_mgop_destroy": [vp],
            "bsgpu_mgop_get_operator": [vp, vp],
            "bsgpu_mgop_read_left_cob": [vp, vp],
            "bsgpu_mgop_add_h_level": [vp, i32, i64, i64, vp, vp, vp],
            "bsgpu_mgop_set_cell_neighbours": [vp, i32, vp],
            "bsgpu_mgop_set_cell_features": [vp, i32, vp],
            "bsgpu_solver_train_learned": [vp, i32, i32, dbl, C.c_uint64, vp],
            "bsgpu_solver_config_default": [vp],
            "bsgpu_solver_create": [vp, vp, vp],
            "bsgpu_solver_destroy": [vp],
            "bsgpu_solver_solve": [vp, vp, vp, vp],
            "bsgpu_solver_solve_device": [vp, vp, vp, vp],
            "bsgpu_solver_get_history": [vp, vp, i32, vp],
            "bsgpu_solver_set_tracing": [vp, i32],
            "bsgpu_solver_get_trace": [vp, C.c_char_p, C.c_size_t],
            "bsgpu_solver_learned_info": [vp, vp],
            "bsgpu_solver_learned_get_weights": [vp, vp, vp, vp],
            "bsgpu_solver_learned_set_weights": [vp, vp, vp, vp],
            "bsgpu_solver_learned_apply": [vp, vp, vp],
            "bsgpu_solver_learned_gradient": [vp, vp, vp, vp, vp, vp],
            "bsgpu_batch_create": [vp, vp, i32],
            "bsgpu_batch_solve_device": [vp, vp, vp, vp],
            "bsgpu_batch_destroy": [vp],
            "bsgpu_assemble_sip_cartesian": [vp, i32, vp, dbl, dbl, i32, dbl, vp, i32],
            "bsgpu_sip_templates": [i32, i32, vp, vp, i64, vp],
            "bsgpu_schwarz_blocks": [i64, vp, vp, i64, i32, vp, vp, vp, vp],
            "bsgpu_ilu_wavefronts": [i64, vp, vp, vp, vp, vp],
            "bsgpu_project_separable": [i32, vp, i32, i32, vp, vp, vp, i32],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(2048)
    lib().bsgpu_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int):
    if rc != OK:
        msg = last_error()
        if rc == ERR_ARGUMENT:
            raise BsgpuArgumentError(rc, msg)
        if rc == ERR_ARITHMETIC:
            raise BsgpuArithmeticError(rc, msg)
        raise BsgpuError(rc, msg)


def launch_count() -> int:
    n = C.c_uint64()
    check(lib().bsgpu_get_launch_count(C.byref(n)))
    return n.value


def ptr(a) -> int:
    """Address of a numpy array or a torch tensor (contiguous)."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def autotune_report():
    """Every launch-shape decision of the autotuner in this process (list of dicts)."""
    import json
    buf = C.create_string_buffer(1 << 20)
    check(lib().bsgpu_autotune_report(buf, len(buf)))
    return json.loads(buf.value.decode())
