"""ctypes binding of oracle/_ref/libpdcs_ref_proj.so: the reference's own cone
projections (src/pdcs_gpu/cuda/massive_block_proj.cu + exp_proj.cu) built as
host code (TEST INFRASTRUCTURE ONLY; tests/ and the golden-fixture script use
it to pin the oracle and the CUDA projections to the reference).

`project(kind, v, S)` maps the oracle's convention -- one block projected onto
S o K = {p : p / S in K} for the per-element scaling S (Dr_product or
Dl_product) -- onto the arrays the reference kernel takes
(preprocess.jl:173-298, def_rpdhg_gen.jl:59): D_scaled = S0/S_i for SOC,
sqrt(S0 S1)/S_i for RSOC, 1/S_i for the dual exponential cone.

Exponential cone (codes 27 and 15): the kernel inverts D_scaled
(massive_block_proj.cu:1184-1190) and exponent_proj_diagonal inverts it again
(exp_proj.cu:777-779), so the host's D_scaled = 1/S (preprocess.jl:223-228)
makes the GPU reference project onto (1/S) o K_exp, while the CPU solver
(exponent_proj_diagonal!, src/pdcs_cpu/exp_proj.jl:682, called with
Dr_product by src/pdcs_cpu/def_rpdhg_gen.jl:42-60) projects onto S o K_exp.
The build follows the CPU solver; to pin the reference kernel's arithmetic on
that same set, D_scaled = S is passed for these codes.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libpdcs_ref_proj.so")
REF_CUDA = "/root/reference/src/pdcs_gpu/cuda"

# reference projection codes (def_rpdhg_gen.jl:265-279): primal-side codes
CODE = {("soc", False): 20, ("soc", True): 22, ("rsoc", False): 23, ("rsoc", True): 25,
        ("exp", False): 26, ("exp", True): 27, ("dexp", False): 28, ("dexp", True): 29}
# the floor the reference's adaptive projection tolerance reaches
# (rpdhg_alg_gpu_gen_scaling.jl:722-723: max(min(tol, kkt * 1e-9, 1e-7), 5e-16))
TOL_FLOOR = 5e-16

_lib = None
_f64p = C.POINTER(C.c_double)
_longp = C.POINTER(C.c_long)


def available():
    return os.path.exists(LIB_PATH) or os.path.isdir(REF_CUDA)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)
        L = C.CDLL(LIB_PATH)
        L.pdcs_ref_block_proj.argtypes = [_f64p] * 8 + [_longp, _longp, C.c_int, _longp, C.c_double, C.c_double]
        L.pdcs_ref_block_proj.restype = C.c_int
        _lib = L
    return _lib


def d_scaled(kind, S):
    S = np.asarray(S, dtype=np.float64)
    if kind == "soc":
        return S[0] / S
    if kind == "rsoc":
        return np.sqrt(S[0] * S[1]) / S
    if kind == "exp":
        return S.copy()
    return 1.0 / S


def project(kind, v, S=None, abs_tol=TOL_FLOOR, rel_tol=TOL_FLOOR, warm=0.0):
    """One block through the reference kernel; returns (projection, warm start after)."""
    arr = np.array(v, dtype=np.float64)
    d = arr.size
    scaled = S is not None
    D = d_scaled(kind, S) if scaled else np.ones(d)
    D2 = D * D
    s1, s2 = np.zeros(d), np.zeros(d)
    tw = np.array([warm], dtype=np.float64)
    head = np.array([0], dtype=np.int64)
    ns = np.array([d], dtype=np.int64)
    code = np.array([CODE[(kind, scaled)]], dtype=np.int64)
    fp = lambda a: a.ctypes.data_as(_f64p)  # noqa: E731
    lp = lambda a: a.ctypes.data_as(_longp)  # noqa: E731
    lib().pdcs_ref_block_proj(fp(arr), fp(arr), fp(arr), fp(D), fp(D2), fp(s1), fp(s2), fp(tw),
                              lp(head), lp(ns), 1, lp(code), abs_tol, rel_tol)
    return arr, float(tw[0])


class Guarded:
    """Runs `project` in a worker process with a per-call time limit.

    Some inputs make the reference's search loops run without end (unbounded
    doubling or bisection loops that never meet their exit test); such a call
    is reported as None and the worker is replaced.  The worker is started
    with `spawn`, so it never inherits a CUDA context."""

    def __init__(self, timeout=2.0):
        import multiprocessing as mp
        self.ctx = mp.get_context("spawn")
        self.timeout = timeout
        self.proc = None
        self.conn = None

    def _start(self):
        a, b = self.ctx.Pipe()
        self.proc = self.ctx.Process(target=_serve, args=(b,), daemon=True)
        self.proc.start()
        self.conn = a

    def project(self, kind, v, S=None):
        if self.proc is None:
            self._start()
        self.conn.send((kind, np.asarray(v, float), None if S is None else np.asarray(S, float)))
        if self.conn.poll(self.timeout):
            return self.conn.recv()
        self.close()
        return None

    def close(self):
        if self.proc is not None:
            self.proc.kill()
            self.proc.join()
            self.proc = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _serve(conn):
    while True:
        try:
            kind, v, S = conn.recv()
        except EOFError:
            return
        conn.send(project(kind, v, S)[0])
