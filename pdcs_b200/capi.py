"""ctypes binding of libpdcs_b200.so (the C ABI declared in include/pdcs.h).

The library is the only compute path: importing this module never falls back
to a CPU implementation, and calling into it without the built library or
without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpdcs_b200.so")

_P = C.POINTER
_vp = C.c_void_p

PDCS_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "m does not match the sum of mGzero, mGnonnegative, socG, rsocG, and (expG + dual_expG) * 3",
    -4: "The size of the SOC must be greater than 1",
    -5: "The size of the rotated SOC must be greater than 2",
    -6: "Not all elements of bl are less than or equal to the corresponding elements in bu",
    -7: "cone blocks of x exceed n",
    -8: "no CUDA device",
    -9: "The combination of options is not supported.",
    -10: "m + nnz exceeds the fixed scratch of pdcs_spmv_csr_noalloc (134217728 merge items)",
}
EXIT_STATUS = {
    0: "optimal", 1: "max_iter", 2: "primal_infeasible_low_acc", 3: "primal_infeasible_high_acc",
    4: "dual_infeasible_low_acc", 5: "dual_infeasible_high_acc", 6: "time_limit", 7: "continue",
    8: "numerical_error_nan", 9: "numerical_error_inf", 10: "attempt_limit",
}


class PdcsProblem(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("nb", C.c_int64), ("nnz", C.c_int64),
                ("G_rowptr", _vp), ("G_colind", _vp), ("G_val", _vp),
                ("c", _vp), ("h", _vp), ("bl", _vp), ("bu", _vp),
                ("mGzero", C.c_int64), ("mGnonnegative", C.c_int64),
                ("socG", _vp), ("n_socG", C.c_int64),
                ("rsocG", _vp), ("n_rsocG", C.c_int64),
                ("expG", C.c_int64), ("dual_expG", C.c_int64),
                ("soc_x", _vp), ("n_soc_x", C.c_int64),
                ("rsoc_x", _vp), ("n_rsoc_x", C.c_int64),
                ("exp_x", C.c_int64), ("dual_exp_x", C.c_int64),
                ("on_device", C.c_int32), ("reserved", C.c_int32)]


class PdcsOptions(C.Structure):
    _fields_ = [("rescaling_method", C.c_int32), ("use_preconditioner", C.c_int32),
                ("use_adaptive_restart", C.c_int32), ("use_adaptive_step_size_weight", C.c_int32),
                ("use_aggressive", C.c_int32), ("use_accelerated", C.c_int32),
                ("use_resolving", C.c_int32), ("warm_start", C.c_int32),
                ("primal_sol", _vp), ("dual_sol", _vp),
                ("max_outer_iter", C.c_int64), ("max_inner_iter", C.c_int64),
                ("abs_tol", C.c_double), ("rel_tol", C.c_double),
                ("eps_primal_infeasible_low_acc", C.c_double), ("eps_dual_infeasible_low_acc", C.c_double),
                ("eps_primal_infeasible_high_acc", C.c_double), ("eps_dual_infeasible_high_acc", C.c_double),
                ("print_freq", C.c_int64), ("check_terminate_freq", C.c_int64),
                ("verbose", C.c_int32), ("use_kkt_restart", C.c_int32),
                ("time_limit", C.c_double), ("kkt_restart_freq", C.c_int64),
                ("use_duality_gap_restart", C.c_int32), ("precision", C.c_int32),
                ("duality_gap_restart_freq", C.c_int64), ("attempt_limit", C.c_int64),
                ("stream", _vp), ("attempts_per_graph", C.c_int32), ("force_resolving", C.c_int32),
                ("spmv_lane_nnz", C.c_int32), ("differentiable", C.c_int32),
                ("spmv_tiles", C.c_int32), ("reserved", C.c_int32)]


class PdcsResult(C.Structure):
    _fields_ = [("x", _vp), ("y", _vp), ("x_device", _vp), ("y_device", _vp),
                ("exit_code", C.c_int32), ("returned_sequence", C.c_int32),
                ("pObj", C.c_double), ("dObj", C.c_double),
                ("iter", C.c_int64), ("restart_used", C.c_int64),
                ("time", C.c_double), ("setup_time", C.c_double),
                ("l_inf_rel_primal_res", C.c_double), ("l_inf_rel_dual_res", C.c_double),
                ("rel_gap", C.c_double), ("l_2_rel_primal_res", C.c_double),
                ("l_2_rel_dual_res", C.c_double), ("l_inf_abs_primal_res", C.c_double),
                ("l_inf_abs_dual_res", C.c_double), ("abs_gap", C.c_double),
                ("kernel_launches", C.c_int64), ("graph_launches", C.c_int64),
                ("time_iterations", C.c_double), ("time_exit_checks", C.c_double),
                ("time_restarts", C.c_double), ("restart_probes", C.c_int64),
                ("spmv_lane_nnz_G", C.c_int32), ("spmv_lane_nnz_Gt", C.c_int32)]


class PdcsBatchInfo(C.Structure):
    _fields_ = [("setup_time", C.c_double), ("solve_time", C.c_double), ("time_iterations", C.c_double),
                ("kernel_launches", C.c_int64), ("graph_launches", C.c_int64),
                ("service_rounds", C.c_int64), ("single_fallbacks", C.c_int64),
                ("spmv_tiled", C.c_int32), ("tail_rounds", C.c_int32)]


class PdcsGradOptions(C.Structure):
    _fields_ = [("rel_tol", C.c_double), ("restart", C.c_int32), ("reserved", C.c_int32),
                ("max_iter", C.c_int64)]


class PdcsGradInfo(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("residual", C.c_double), ("time", C.c_double),
                ("converged", C.c_int32), ("reserved", C.c_int32)]


# every symbol declared in include/pdcs.h
EXPORTS = ["pdcs_default_options", "pdcs_solve", "pdcs_solve_batch", "pdcs_batch_create", "pdcs_batch_solve",
           "pdcs_batch_destroy", "pdcs_batch_grad", "pdcs_grad", "pdcs_block_proj", "pdcs_spmv_csr",
           "pdcs_spmv_csr_noalloc", "pdcs_version"]

_lib = None


def load():
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m pdcs_b200.build` "
                           "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.pdcs_default_options.argtypes = [_P(PdcsOptions)]
    L.pdcs_default_options.restype = C.c_int
    L.pdcs_solve.argtypes = [_P(PdcsProblem), _P(PdcsOptions), _P(PdcsResult)]
    L.pdcs_solve.restype = C.c_int
    L.pdcs_solve_batch.argtypes = [C.c_int64, _P(PdcsProblem), _P(PdcsOptions), _P(PdcsResult), _P(PdcsBatchInfo)]
    L.pdcs_solve_batch.restype = C.c_int
    L.pdcs_batch_create.argtypes = [C.c_int64, _P(PdcsProblem), _P(PdcsOptions), _P(_vp)]
    L.pdcs_batch_create.restype = C.c_int
    L.pdcs_batch_solve.argtypes = [_vp, C.c_int64, _P(PdcsResult), _P(PdcsBatchInfo)]
    L.pdcs_batch_solve.restype = C.c_int
    L.pdcs_batch_destroy.argtypes = [_vp]
    L.pdcs_batch_destroy.restype = None
    _pp = _P(_vp)
    L.pdcs_batch_grad.argtypes = [_vp, _pp, _pp, _pp, _pp, _pp, _pp, _pp, _P(PdcsGradOptions), _P(PdcsGradInfo)]
    L.pdcs_batch_grad.restype = C.c_int
    L.pdcs_grad.argtypes = [_P(PdcsProblem), _P(PdcsOptions), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                            _P(PdcsGradOptions), _P(PdcsGradInfo)]
    L.pdcs_grad.restype = C.c_int
    L.pdcs_block_proj.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, C.c_int64, _vp, _vp]
    L.pdcs_block_proj.restype = C.c_int
    L.pdcs_spmv_csr.argtypes = [C.c_int64, C.c_int64, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp]
    L.pdcs_spmv_csr.restype = C.c_int
    L.pdcs_spmv_csr_noalloc.argtypes = [C.c_int64, C.c_int64, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp]
    L.pdcs_spmv_csr_noalloc.restype = C.c_int
    L.pdcs_version.restype = C.c_char_p
    _lib = L
    return L


def check(rc, what="pdcs"):
    if rc != PDCS_OK:
        raise RuntimeError(f"{what} failed: {ERRORS.get(rc, rc)} (status {rc})")
