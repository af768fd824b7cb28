"""ctypes binding of the CPU oracle (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpdcs_oracle.so")

KIND = dict(free=0, zero=1, nonneg=2, box=3, soc=4, rsoc=5, exp=6, dexp=7)

_P = C.POINTER
_i64p = _P(C.c_int64)
_f64p = _P(C.c_double)


class OracleProblem(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("nb", C.c_int64), ("nnz", C.c_int64),
                ("rowptr", _i64p), ("colind", _i64p), ("val", _f64p),
                ("c", _f64p), ("h", _f64p), ("bl", _f64p), ("bu", _f64p),
                ("mGzero", C.c_int64), ("mGnonneg", C.c_int64),
                ("socG", _i64p), ("n_socG", C.c_int64),
                ("rsocG", _i64p), ("n_rsocG", C.c_int64),
                ("expG", C.c_int64), ("dual_expG", C.c_int64),
                ("soc_x", _i64p), ("n_soc_x", C.c_int64),
                ("rsoc_x", _i64p), ("n_rsoc_x", C.c_int64),
                ("exp_x", C.c_int64), ("dual_exp_x", C.c_int64)]


class OracleOptions(C.Structure):
    _fields_ = [("max_outer_iter", C.c_int64), ("max_inner_iter", C.c_int64),
                ("abs_tol", C.c_double), ("rel_tol", C.c_double),
                ("eps_primal_infeasible_low_acc", C.c_double),
                ("eps_dual_infeasible_low_acc", C.c_double),
                ("eps_primal_infeasible_high_acc", C.c_double),
                ("eps_dual_infeasible_high_acc", C.c_double),
                ("check_terminate_freq", C.c_int64), ("kkt_restart_freq", C.c_int64),
                ("duality_gap_restart_freq", C.c_int64),
                ("use_kkt_restart", C.c_int32), ("use_duality_gap_restart", C.c_int32),
                ("rescaling", C.c_int32), ("cpu_semantics", C.c_int32),
                ("threads", C.c_int32), ("verbose", C.c_int32),
                ("time_limit", C.c_double), ("attempt_limit", C.c_int64),
                ("warm_x", _f64p), ("warm_y", _f64p),
                ("force_resolving", C.c_int32), ("pad", C.c_int32)]


class OracleResult(C.Structure):
    _fields_ = [("x", _f64p), ("y", _f64p),
                ("primal_objective", C.c_double), ("dual_objective", C.c_double),
                ("l_inf_rel_primal_res", C.c_double), ("l_inf_rel_dual_res", C.c_double),
                ("rel_gap", C.c_double), ("l_2_rel_primal_res", C.c_double),
                ("l_2_rel_dual_res", C.c_double), ("iter", C.c_int64),
                ("restart_used", C.c_int64), ("exit_code", C.c_int32),
                ("returned_sequence", C.c_int32), ("solve_seconds", C.c_double),
                ("setup_seconds", C.c_double)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oracle_default_options.argtypes = [_P(OracleOptions)]
        L.oracle_project_block.argtypes = [C.c_int, _f64p, C.c_int64, _f64p, _f64p, _f64p]
        L.oracle_project_block.restype = C.c_int
        L.oracle_proj_exp_scaled.argtypes = [_f64p, _f64p]
        L.oracle_solve.argtypes = [_P(OracleProblem), _P(OracleOptions), _P(OracleResult)]
        L.oracle_solve.restype = C.c_int
        L.oracle_precondition.argtypes = [_P(OracleProblem), C.c_int, _f64p, _f64p, _f64p]
        L.oracle_precondition.restype = C.c_int
        L.oracle_evaluate.argtypes = [_P(OracleProblem), _f64p, _f64p, _f64p]
        L.oracle_evaluate.restype = C.c_int
        _lib = L
    return _lib


def _f(a):
    return a.ctypes.data_as(_f64p) if a is not None and a.size else None


def _i(a):
    return a.ctypes.data_as(_i64p) if a is not None and a.size else None


def project_block(kind, v, S=None, lo=None, hi=None):
    """Project one block (returns a new array)."""
    k = KIND[kind] if isinstance(kind, str) else int(kind)
    out = np.ascontiguousarray(v, dtype=np.float64).copy()
    S = None if S is None else np.ascontiguousarray(S, dtype=np.float64)
    lo = None if lo is None else np.ascontiguousarray(lo, dtype=np.float64)
    hi = None if hi is None else np.ascontiguousarray(hi, dtype=np.float64)
    rc = lib().oracle_project_block(k, _f(out), out.size, _f(S), _f(lo), _f(hi))
    if rc != 0:
        raise ValueError(f"oracle_project_block rc={rc}")
    return out


class _Keep:
    """Holds numpy buffers alive while a ctypes struct points at them."""

    def __init__(self):
        self.bufs = []

    def f(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.bufs.append(a)
        return _f(a)

    def i(self, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.int64))
        self.bufs.append(a)
        return _i(a)


def _problem_struct(prob, keep):
    G = prob.G.tocsr()
    P = OracleProblem()
    P.n, P.m, P.nb, P.nnz = prob.n, prob.m, prob.nb, G.nnz
    P.rowptr = keep.i(G.indptr)
    P.colind = keep.i(G.indices)
    P.val = keep.f(G.data)
    P.c, P.h = keep.f(prob.c), keep.f(prob.h)
    P.bl, P.bu = keep.f(prob.bl), keep.f(prob.bu)
    P.mGzero, P.mGnonneg = prob.mGzero, prob.mGnonnegative
    P.socG, P.n_socG = keep.i(prob.socG), len(prob.socG)
    P.rsocG, P.n_rsocG = keep.i(prob.rsocG), len(prob.rsocG)
    P.expG, P.dual_expG = prob.expG, prob.dual_expG
    P.soc_x, P.n_soc_x = keep.i(prob.soc_x), len(prob.soc_x)
    P.rsoc_x, P.n_rsoc_x = keep.i(prob.rsoc_x), len(prob.rsoc_x)
    P.exp_x, P.dual_exp_x = prob.exp_x, prob.dual_exp_x
    return P


def solve(prob, **opts):
    """Run the oracle solver; returns a dict with x, y and the info fields."""
    keep = _Keep()
    P = _problem_struct(prob, keep)
    O = OracleOptions()
    lib().oracle_default_options(C.byref(O))
    for k, v in opts.items():
        if k in ("warm_x", "warm_y"):
            setattr(O, k, keep.f(v))
        elif k == "rescaling_method":
            O.rescaling = {"none": 0, "ruiz": 1, "pock_chambolle": 2, "ruiz_pock_chambolle": 3}[v]
        else:
            setattr(O, k, v)
    x = np.zeros(prob.n)
    y = np.zeros(prob.m)
    R = OracleResult()
    R.x, R.y = _f(x), _f(y)
    rc = lib().oracle_solve(C.byref(P), C.byref(O), C.byref(R))
    if rc != 0:
        raise ValueError(f"oracle_solve rc={rc}")
    out = {k: getattr(R, k) for k, _ in OracleResult._fields_ if k not in ("x", "y")}
    out["x"], out["y"] = x, y
    return out


def precondition(prob, rescaling=3):
    keep = _Keep()
    P = _problem_struct(prob, keep)
    Dr = np.zeros(prob.n)
    Dl = np.zeros(prob.m)
    val = np.zeros(prob.G.nnz)
    rc = lib().oracle_precondition(C.byref(P), rescaling, _f(Dr), _f(Dl), _f(val))
    if rc != 0:
        raise ValueError(f"oracle_precondition rc={rc}")
    return Dr, Dl, val


EVAL_KEYS = ("primal_res", "dual_res", "rel_gap", "primal_res_gpu_form", "pobj", "dobj",
             "primal_abs_inf", "dual_abs_inf")


def evaluate(prob, x, y):
    """Score a final point with the shared FP64 evaluator (README-form criteria)."""
    keep = _Keep()
    P = _problem_struct(prob, keep)
    out = np.zeros(8)
    xv = np.ascontiguousarray(x, dtype=np.float64)
    yv = np.ascontiguousarray(y, dtype=np.float64)
    rc = lib().oracle_evaluate(C.byref(P), _f(xv), _f(yv), _f(out))
    if rc != 0:
        raise ValueError(f"oracle_evaluate rc={rc}")
    d = dict(zip(EVAL_KEYS, out.tolist()))
    d["max_rel"] = max(d["primal_res"], d["dual_res"], d["rel_gap"])
    return d
