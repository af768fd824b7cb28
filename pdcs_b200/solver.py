"""Python front-end mirroring PDCS's solver entry point.

``rpdhg_gpu_solve`` takes the keyword arguments of the reference's
``rpdhg_gpu_solve`` (src/pdcs_gpu/rpdhg_alg_gpu_gen.jl:1219-1268) and returns a
``Solution`` whose fields follow the ones the reference's wrappers read
(``x.recovered_primal.primal_sol.x``, ``y.recovered_dual.dual_sol.y``,
``info.exit_status`` / ``exit_code`` / ``pObj`` / ``dObj`` / ``iter`` / ``time``,
src/pdcs_gpu/MOI_wrapper/MOI_wrapper.jl:648-658).  Validation errors raise
like the reference (rpdhg_alg_gpu_gen.jl:1331-1375, :84, :94).

Inputs may be numpy / scipy (copied to the device by the library) or CUDA
torch tensors (used in place, zero copy).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from types import SimpleNamespace
from typing import Optional, Sequence

import numpy as np
import scipy.sparse as sp

from . import capi

_RESCALING = {"none": 0, "ruiz": 1, "pock_chambolle": 2, "ruiz_pock_chambolle": 3}


@dataclasses.dataclass
class Info:
    exit_status: str
    exit_code: int
    pObj: float
    dObj: float
    iter: int
    time: float
    setup_time: float
    restart_used: int
    l_inf_rel_primal_res: float
    l_inf_rel_dual_res: float
    rel_gap: float
    l_2_rel_primal_res: float
    l_2_rel_dual_res: float
    l_inf_abs_primal_res: float
    l_inf_abs_dual_res: float
    abs_gap: float
    returned_sequence: int
    kernel_launches: int
    graph_launches: int
    time_iterations: float = 0.0
    time_exit_checks: float = 0.0
    time_restarts: float = 0.0
    restart_probes: int = 0
    spmv_lane_nnz: tuple = (0, 0)


class Solution:
    """Result of a solve; ``x`` / ``y`` are the recovered (original-scale) vectors."""

    def __init__(self, x, y, info: Info):
        self.x = SimpleNamespace(recovered_primal=SimpleNamespace(primal_sol=SimpleNamespace(x=x)))
        self.y = SimpleNamespace(recovered_dual=SimpleNamespace(dual_sol=SimpleNamespace(y=y)))
        self.info = info
        self.primal = x
        self.dual = y

    def __repr__(self):
        i = self.info
        return (f"Solution(exit_status={i.exit_status}, iter={i.iter}, pObj={i.pObj:.10g}, "
                f"dObj={i.dObj:.10g}, time={i.time:.4f}s)")


def _is_torch_cuda(a):
    return type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False)


class _Holder:
    """Keeps host buffers alive and returns raw pointers for the C struct."""

    def __init__(self):
        self.keep = []

    def f64(self, a):
        if a is None:
            return None
        if _is_torch_cuda(a):
            import torch
            a = a.to(torch.float64).contiguous()
            self.keep.append(a)
            return a.data_ptr()
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        self.keep.append(a)
        return a.ctypes.data if a.size else None

    def i32(self, a):
        if _is_torch_cuda(a):
            import torch
            a = a.to(torch.int32).contiguous()
            self.keep.append(a)
            return a.data_ptr()
        a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
        self.keep.append(a)
        return a.ctypes.data if a.size else None

    def i64(self, a):
        a = np.ascontiguousarray(np.asarray(a if isinstance(a, np.ndarray) else list(a), dtype=np.int64).reshape(-1))
        self.keep.append(a)
        return a.ctypes.data if a.size else None


_PROBLEM_KEYS = ("n", "m", "nb", "c", "G", "h", "mGzero", "mGnonnegative", "socG", "rsocG", "expG",
                 "dual_expG", "bl", "bu", "soc_x", "rsoc_x", "exp_x", "dual_exp_x", "Dl", "Dr")


def _problem_struct(hold: _Holder, *, n, m, nb, c, G, h, mGzero, mGnonnegative, socG, rsocG, expG, dual_expG,
                    bl, bu, soc_x, rsoc_x, exp_x=0, dual_exp_x=0, Dl=None, Dr=None):
    """Validate like the reference (rpdhg_alg_gpu_gen.jl:1331-1375, :84, :94) and fill a PdcsProblem."""
    on_device = _is_torch_cuda(c)
    if not on_device:
        if not (sp.issparse(G) and G.format == "csr"):
            G = sp.csr_matrix(G)
        if not G.has_sorted_indices:  # scipy caches the check on the matrix; repeated solves skip the scan
            G = G.sorted_indices()  # a sorted copy: the caller's arrays are never reordered
        if G.shape[0] != m:
            raise ValueError("m does not match the size of G")
        if G.shape[1] != n:
            raise ValueError("n does not match the size of G")
        rowptr, colind, val = G.indptr, G.indices, G.data
        nnz = G.nnz
        bl = np.asarray(bl, dtype=np.float64)
        bu = np.asarray(bu, dtype=np.float64)
        if bl.shape != (nb,) or bu.shape != (nb,):
            raise ValueError("bl and bu must have length nb")
        if not np.all(bl <= bu):
            raise ValueError("Not all elements of bl are less than or equal to the corresponding elements in bu")
    else:
        rowptr, colind, val = G  # (crow_indices, col_indices, values) tensors on the device
        nnz = int(val.numel())
    socG, rsocG, soc_x, rsoc_x = (np.asarray(d, dtype=np.int64).reshape(-1) for d in (socG, rsocG, soc_x, rsoc_x))
    if m != mGzero + mGnonnegative + int(socG.sum()) + int(rsocG.sum()) + (expG + dual_expG) * 3:
        raise ValueError("m does not match the sum of mGzero, mGnonnegative, socG, rsocG, "
                         "and (expG + dual_expG) * 3")
    if (socG.size and socG.min() < 2) or (soc_x.size and soc_x.min() < 2):
        raise ValueError("The size of the SOC must be greater than 1")
    if (rsocG.size and rsocG.min() < 3) or (rsoc_x.size and rsoc_x.min() < 3):
        raise ValueError("The size of the rotated SOC must be greater than 2")
    P = capi.PdcsProblem()
    P.n, P.m, P.nb, P.nnz = n, m, nb, nnz
    P.G_rowptr, P.G_colind, P.G_val = hold.i32(rowptr), hold.i32(colind), hold.f64(val)
    P.c, P.h, P.bl, P.bu = hold.f64(c), hold.f64(h), hold.f64(bl), hold.f64(bu)
    P.mGzero, P.mGnonnegative = mGzero, mGnonnegative
    P.socG, P.n_socG = hold.i64(socG), len(socG)
    P.rsocG, P.n_rsocG = hold.i64(rsocG), len(rsocG)
    P.expG, P.dual_expG = expG, dual_expG
    P.soc_x, P.n_soc_x = hold.i64(soc_x), len(soc_x)
    P.rsoc_x, P.n_rsoc_x = hold.i64(rsoc_x), len(rsoc_x)
    P.exp_x, P.dual_exp_x = exp_x, dual_exp_x
    P.on_device = 1 if on_device else 0
    return P


def _options_struct(L, hold: _Holder, *, n=0, m=0, rescaling_method: str = "ruiz_pock_chambolle",
                    use_preconditioner: bool = True, use_adaptive_restart: bool = True,
                    use_adaptive_step_size_weight: bool = True, use_aggressive: bool = True,
                    use_accelerated: bool = False, use_resolving: bool = True, primal_sol=None, dual_sol=None,
                    warm_start: bool = False, max_outer_iter: int = 10000, max_inner_iter: int = 500000,
                    abs_tol: float = 1e-6, rel_tol: float = 1e-6, eps_primal_infeasible_low_acc: float = 1e-12,
                    eps_dual_infeasible_low_acc: float = 1e-12, eps_primal_infeasible_high_acc: float = 1e-16,
                    eps_dual_infeasible_high_acc: float = 1e-16, print_freq: int = 2000,
                    check_terminate_freq: int = 2000, verbose: int = 0, time_limit: float = math.inf,
                    method: str = "average", logfile_name: Optional[str] = None, use_kkt_restart: bool = False,
                    kkt_restart_freq: int = 2000, use_duality_gap_restart: bool = True,
                    duality_gap_restart_freq: int = 2000, attempt_limit: int = 0, attempts_per_graph: int = 32,
                    stream=None, force_resolving: bool = False, precision="fp64", spmv_lane_nnz: int = 0,
                    differentiable: bool = False, spmv_tiles=True):
    """Fill a PdcsOptions from the reference's keyword arguments (rpdhg_alg_gpu_gen.jl:1219-1268).

    precision: "fp64" (the reference's arithmetic) or "fp32" (FP32 matrices and iterate deltas
    between FP64 anchors; FP64 projections, averages and termination checks).
    spmv_lane_nnz: 0 autotunes the SpMV schedule per matrix; 1..16 fixes it (nonzeros per lane).
    spmv_tiles: batched solves run the instance-tiled SpMV (instance column segments staged in
    shared memory) when every instance fits it; False keeps the binned row schedule; an int
    sets the nonzeros per tile."""
    if method not in ("average", "halpern"):
        raise ValueError("method only available for :average and :halpern")
    if method == "halpern":
        raise NotImplementedError("method=:halpern is not wired into the reference GPU module either")
    if warm_start and (primal_sol is None or dual_sol is None or len(primal_sol) != n or len(dual_sol) != m):
        raise ValueError("Warmstart doesn't match the problem size")
    O = capi.PdcsOptions()
    L.pdcs_default_options(C.byref(O))
    O.rescaling_method = _RESCALING[rescaling_method.lstrip(":")]
    O.use_preconditioner = int(use_preconditioner)
    O.use_adaptive_restart = int(use_adaptive_restart)
    O.use_adaptive_step_size_weight = int(use_adaptive_step_size_weight)
    O.use_aggressive = int(use_aggressive)
    O.use_accelerated = int(use_accelerated)
    O.use_resolving = int(use_resolving)
    O.warm_start = int(warm_start)
    if warm_start:
        O.primal_sol = hold.f64(np.asarray(primal_sol, dtype=np.float64))
        O.dual_sol = hold.f64(np.asarray(dual_sol, dtype=np.float64))
    O.max_outer_iter, O.max_inner_iter = max_outer_iter, max_inner_iter
    O.abs_tol, O.rel_tol = abs_tol, rel_tol
    O.eps_primal_infeasible_low_acc = eps_primal_infeasible_low_acc
    O.eps_dual_infeasible_low_acc = eps_dual_infeasible_low_acc
    O.eps_primal_infeasible_high_acc = eps_primal_infeasible_high_acc
    O.eps_dual_infeasible_high_acc = eps_dual_infeasible_high_acc
    O.print_freq, O.check_terminate_freq = print_freq, check_terminate_freq
    O.verbose = int(verbose)
    O.use_kkt_restart = int(use_kkt_restart)
    O.time_limit = 0.0 if not math.isfinite(time_limit) else float(time_limit)
    O.kkt_restart_freq = kkt_restart_freq
    O.use_duality_gap_restart = int(use_duality_gap_restart)
    O.duality_gap_restart_freq = duality_gap_restart_freq
    O.attempt_limit = attempt_limit
    O.attempts_per_graph = attempts_per_graph
    O.force_resolving = int(force_resolving)
    O.stream = stream
    prec = {"fp64": 0, "fp32": 1, 0: 0, 1: 1}.get(precision)
    if prec is None:
        raise ValueError("precision must be 'fp64' or 'fp32'")
    O.precision = prec
    if spmv_lane_nnz not in (0, 1, 2, 4, 8, 16):
        raise ValueError("spmv_lane_nnz must be 0 (autotune) or a power of two up to 16")
    O.spmv_lane_nnz = spmv_lane_nnz
    O.differentiable = int(differentiable)
    if spmv_tiles is True or spmv_tiles is False:
        O.spmv_tiles = 0 if spmv_tiles else -1
    elif int(spmv_tiles) > 0:
        O.spmv_tiles = int(spmv_tiles)
    else:
        raise ValueError("spmv_tiles must be True, False or a positive number of nonzeros per tile")
    return O


def _info(R) -> Info:
    return Info(exit_status=capi.EXIT_STATUS.get(R.exit_code, str(R.exit_code)),
                exit_code=R.exit_code, pObj=R.pObj, dObj=R.dObj, iter=R.iter, time=R.time,
                setup_time=R.setup_time, restart_used=R.restart_used,
                l_inf_rel_primal_res=R.l_inf_rel_primal_res,
                l_inf_rel_dual_res=R.l_inf_rel_dual_res, rel_gap=R.rel_gap,
                l_2_rel_primal_res=R.l_2_rel_primal_res, l_2_rel_dual_res=R.l_2_rel_dual_res,
                l_inf_abs_primal_res=R.l_inf_abs_primal_res,
                l_inf_abs_dual_res=R.l_inf_abs_dual_res, abs_gap=R.abs_gap,
                returned_sequence=R.returned_sequence, kernel_launches=R.kernel_launches,
                graph_launches=R.graph_launches, time_iterations=R.time_iterations,
                time_exit_checks=R.time_exit_checks, time_restarts=R.time_restarts,
                restart_probes=R.restart_probes, spmv_lane_nnz=(R.spmv_lane_nnz_G, R.spmv_lane_nnz_Gt))


def rpdhg_gpu_solve(*, device_output: bool = False, **kw) -> Solution:
    """Solve min c'x s.t. Gx - h in K_d, bl <= x[:nb] <= bu, x[nb:] in K_p on the GPU.

    Keywords: the reference's problem data and options (rpdhg_alg_gpu_gen.jl:1219-1268), plus
    attempt_limit, attempts_per_graph, stream, force_resolving and device_output."""
    L = capi.load()
    hold = _Holder()
    P = _problem_struct(hold, **{k: v for k, v in kw.items() if k in _PROBLEM_KEYS})
    O = _options_struct(L, hold, **{k: v for k, v in kw.items() if k not in _PROBLEM_KEYS or k in ("n", "m")})
    n, m = P.n, P.m
    R = capi.PdcsResult()
    if device_output:
        import torch
        xo = torch.empty(n, dtype=torch.float64, device="cuda")
        yo = torch.empty(m, dtype=torch.float64, device="cuda")
        R.x_device, R.y_device = xo.data_ptr(), yo.data_ptr()
    else:
        xo = np.zeros(n)
        yo = np.zeros(m)
        R.x, R.y = (xo.ctypes.data if n else None), (yo.ctypes.data if m else None)
    rc = L.pdcs_solve(C.byref(P), C.byref(O), C.byref(R))
    capi.check(rc, "pdcs_solve")
    return Solution(xo, yo, _info(R))


@dataclasses.dataclass
class BatchInfo:
    setup_time: float
    solve_time: float
    time_iterations: float
    kernel_launches: int
    graph_launches: int
    service_rounds: int
    single_fallbacks: int
    spmv_tiled: bool = False
    tail_rounds: int = 0


class BatchHandle:
    """A prepared batch (pdcs_batch_create): merged, uploaded and preconditioned once;
    ``solve()`` runs a cold-start batched solve of it (pdcs_batch_solve)."""

    def __init__(self, problems, **options):
        self._L = capi.load()
        self._hold = _Holder()
        self._h = C.c_void_p()
        probs = [p.kwargs() if hasattr(p, "kwargs") else dict(p) for p in problems]
        if not probs:
            raise ValueError("empty batch")
        self._Ps = (capi.PdcsProblem * len(probs))()
        for i, kw in enumerate(probs):
            self._Ps[i] = _problem_struct(self._hold, **{k: v for k, v in kw.items() if k in _PROBLEM_KEYS})
            if self._Ps[i].on_device:
                raise ValueError("pdcs_batch_create takes host data")
        self._O = _options_struct(self._L, self._hold, **options)
        self.count = len(probs)
        self.sizes = [(P.n, P.m) for P in self._Ps]
        rc = self._L.pdcs_batch_create(self.count, self._Ps, C.byref(self._O), C.byref(self._h))
        capi.check(rc, "pdcs_batch_create")

    def solve(self, attempt_limit: int = 0):
        """Returns (list of Solution, BatchInfo)."""
        if not self._h:
            raise RuntimeError("batch handle is closed")
        Rs = (capi.PdcsResult * self.count)()
        outs = []
        for i, (n, m) in enumerate(self.sizes):
            xo, yo = np.zeros(n), np.zeros(m)
            outs.append((xo, yo))
            Rs[i].x = xo.ctypes.data if n else None
            Rs[i].y = yo.ctypes.data if m else None
        B = capi.PdcsBatchInfo()
        rc = self._L.pdcs_batch_solve(self._h, attempt_limit, Rs, C.byref(B))
        capi.check(rc, "pdcs_batch_solve")
        return [Solution(outs[i][0], outs[i][1], _info(Rs[i])) for i in range(self.count)], _batch_info(B)

    def grad(self, dldx, dldy=None, rel_tol=1e-10, restart=100, max_iter=5000):
        """Solution-map adjoint at the last solve (the handle must be created with
        differentiable=True).  dldx / dldy: per-instance loss gradients w.r.t. x*, y*
        (dldy may be None).  Returns (list of dicts c, h, G, bl, bu -- G in the
        instance's CSR order with sorted indices --, list of GradInfo)."""
        if not self._h:
            raise RuntimeError("batch handle is closed")
        K = self.count
        keep = []

        def ptrs(arrays, sizes):
            out = (C.c_void_p * K)()
            for i in range(K):
                a = None if arrays is None else arrays[i]
                if a is None:
                    out[i] = None
                    continue
                a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
                if a.shape != (sizes[i],):
                    raise ValueError(f"instance {i}: expected {sizes[i]} values")
                keep.append(a)
                out[i] = a.ctypes.data if a.size else None
            return out
        ns = [n for n, _ in self.sizes]
        ms = [m for _, m in self.sizes]
        nnzs = [P.nnz for P in self._Ps]
        nbs = [P.nb for P in self._Ps]
        res = [dict(c=np.zeros(ns[i]), h=np.zeros(ms[i]), G=np.zeros(nnzs[i]), bl=np.zeros(nbs[i]),
                    bu=np.zeros(nbs[i])) for i in range(K)]
        outs = {}
        for key in ("c", "h", "G", "bl", "bu"):
            outs[key] = (C.c_void_p * K)(*[res[i][key].ctypes.data if res[i][key].size else None for i in range(K)])
        go = capi.PdcsGradOptions(rel_tol=rel_tol, restart=restart, max_iter=max_iter)
        infos = (capi.PdcsGradInfo * K)()
        rc = self._L.pdcs_batch_grad(self._h, ptrs(dldx, ns), ptrs(dldy, ms), outs["c"], outs["h"], outs["G"],
                                     outs["bl"], outs["bu"], C.byref(go), infos)
        capi.check(rc, "pdcs_batch_grad")
        return res, [GradInfo(i.iterations, i.residual, i.time, bool(i.converged)) for i in infos]

    def close(self):
        if self._h:
            self._L.pdcs_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclasses.dataclass
class GradInfo:
    iterations: int
    residual: float
    time: float
    converged: bool


def rpdhg_gpu_grad(problem, x, y, dldx, dldy=None, rel_tol=1e-10, restart=100, max_iter=5000, **options):
    """Solution-map adjoint of one problem at the solution (x, y) (pdcs_grad): returns
    (dict of dL/dc, dL/dh, dL/dG (nonzero values, CSR order with sorted indices), dL/dbl,
    dL/dbu; GradInfo)."""
    L = capi.load()
    hold = _Holder()
    kw = problem.kwargs() if hasattr(problem, "kwargs") else dict(problem)
    P = _problem_struct(hold, **{k: v for k, v in kw.items() if k in _PROBLEM_KEYS})
    O = _options_struct(L, hold, **options)
    out = dict(c=np.zeros(P.n), h=np.zeros(P.m), G=np.zeros(P.nnz), bl=np.zeros(P.nb), bu=np.zeros(P.nb))
    ptr = lambda a: a.ctypes.data if a.size else None
    go = capi.PdcsGradOptions(rel_tol=rel_tol, restart=restart, max_iter=max_iter)
    info = capi.PdcsGradInfo()
    rc = L.pdcs_grad(C.byref(P), C.byref(O), hold.f64(x), hold.f64(y), hold.f64(dldx),
                     None if dldy is None else hold.f64(dldy), ptr(out["c"]), ptr(out["h"]), ptr(out["G"]),
                     ptr(out["bl"]), ptr(out["bu"]), C.byref(go), C.byref(info))
    capi.check(rc, "pdcs_grad")
    return out, GradInfo(info.iterations, info.residual, info.time, bool(info.converged))


def _batch_info(B) -> "BatchInfo":
    return BatchInfo(setup_time=B.setup_time, solve_time=B.solve_time, time_iterations=B.time_iterations,
                     kernel_launches=B.kernel_launches, graph_launches=B.graph_launches,
                     service_rounds=B.service_rounds, single_fallbacks=B.single_fallbacks,
                     spmv_tiled=bool(B.spmv_tiled), tail_rounds=B.tail_rounds)


def rpdhg_gpu_solve_batch(problems, **options):
    """Solve many independent programs in one batched run (pdcs_solve_batch).

    problems: sequence of dicts of rpdhg_gpu_solve's problem keywords (n, m, nb, c, G, h, cones, bl, bu)
    or objects with a ``kwargs()`` method.  options: rpdhg_gpu_solve's option keywords, shared by all
    instances.  Returns (list of Solution, BatchInfo)."""
    L = capi.load()
    hold = _Holder()
    probs = [p.kwargs() if hasattr(p, "kwargs") else dict(p) for p in problems]
    if not probs:
        raise ValueError("empty batch")
    Ps = (capi.PdcsProblem * len(probs))()
    for i, kw in enumerate(probs):
        Ps[i] = _problem_struct(hold, **{k: v for k, v in kw.items() if k in _PROBLEM_KEYS})
        if Ps[i].on_device:
            raise ValueError("pdcs_solve_batch takes host data")
    O = _options_struct(L, hold, **options)
    Rs = (capi.PdcsResult * len(probs))()
    outs = []
    for i, kw in enumerate(probs):
        xo, yo = np.zeros(Ps[i].n), np.zeros(Ps[i].m)
        outs.append((xo, yo))
        Rs[i].x = xo.ctypes.data if Ps[i].n else None
        Rs[i].y = yo.ctypes.data if Ps[i].m else None
    B = capi.PdcsBatchInfo()
    rc = L.pdcs_solve_batch(len(probs), Ps, C.byref(O), Rs, C.byref(B))
    capi.check(rc, "pdcs_solve_batch")
    sols = [Solution(outs[i][0], outs[i][1], _info(Rs[i])) for i in range(len(probs))]
    return sols, _batch_info(B)


def solve_problem(prob, **kw) -> Solution:
    """Convenience: solve a pdcs_b200.problems.ConicProblem."""
    return rpdhg_gpu_solve(**prob.kwargs(), **kw)


def block_proj(arr, codes, head_start, ns, S=None, bl=None, bu=None, stream=None):
    """Project blocks of a CUDA float64 tensor in place (pdcs_block_proj)."""
    import torch
    dev = arr.device
    assert arr.is_cuda and arr.dtype == torch.float64 and arr.is_contiguous()
    hs = torch.as_tensor(np.asarray(head_start, dtype=np.int64), device=dev)
    nn = torch.as_tensor(np.asarray(ns, dtype=np.int64), device=dev)
    cc = torch.as_tensor(np.asarray(codes, dtype=np.int64), device=dev)
    ptr = lambda t: None if t is None else t.data_ptr()
    rc = capi.load().pdcs_block_proj(arr.data_ptr(), ptr(bl), ptr(bu), ptr(S), hs.data_ptr(),
                                     nn.data_ptr(), len(codes), cc.data_ptr(), stream)
    capi.check(rc, "pdcs_block_proj")
    return arr
