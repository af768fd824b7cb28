"""Batched solver (pdcs_solve_batch): every instance follows the single-instance
algorithm with its own step sizes, restarts and termination.

Parity: (1) after a fixed number of attempts each instance's iterates equal the
oracle's to rounding; (2) solved to 1e-6, each instance matches the
single-instance GPU solve (status, objective) and the oracle's evaluator."""
import numpy as np
import pytest

from oracle import binding as B
from _parity import assert_objective
from pdcs_b200 import problems, solver

pytestmark = pytest.mark.gpu


def _mixed_batch():
    return [
        problems.mixed_small(seed=7),
        problems.batch_socp_c3(count=3, seed=11, nmin=50, nmax=400)[0],
        problems.logreg_exp_c1(samples=120, features=12, density=0.3),
        problems.mixed_small(seed=9, scale=2),
        problems.socp_c0(n_box=60, n_soc=60, m=90, density=0.08, seed=5),
    ]


@pytest.mark.parametrize("attempts", [1, 7, 60])
def test_batch_first_attempts_track_oracle(cuda, attempts):
    batch = _mixed_batch()
    sols, info = solver.rpdhg_gpu_solve_batch(batch, attempt_limit=attempts)
    assert info.single_fallbacks == 0
    for p, g in zip(batch, sols):
        o = B.solve(p, threads=1, attempt_limit=attempts)
        assert g.info.exit_code == 10 and o["exit_code"] == 10
        assert g.info.iter == o["iter"] == attempts
        for a, b in ((g.primal, o["x"]), (g.dual, o["y"])):
            scale = max(1.0, np.abs(b).max())
            assert np.abs(a - b).max() <= 1e-9 * scale, (p.name, attempts, np.abs(a - b).max())


def test_batch_matches_single_solves(cuda):
    batch = _mixed_batch() + problems.batch_socp_c3(count=6, seed=23, nmin=50, nmax=600)
    sols, info = solver.rpdhg_gpu_solve_batch(batch, time_limit=300)
    assert info.graph_launches > 0 and info.service_rounds > 0
    for p, g in zip(batch, sols):
        s = solver.solve_problem(p, time_limit=120)
        assert g.info.exit_status == s.info.exit_status == "optimal", (p.name, g, s)
        e = B.evaluate(p, g.primal, g.dual)
        assert max(e["primal_res_gpu_form"], e["dual_res"], e["rel_gap"]) < 1.05e-6, (p.name, e)
        assert abs(g.info.pObj - e["pobj"]) <= 1e-9 * (1 + abs(e["pobj"]))
        assert_objective(p, g.info.pObj, "batch")
        assert_objective(p, s.info.pObj, "single")
        # same algorithm; only the order of floating-point sums differs, which can move
        # convergence across one exit check (every 2000 attempts) or a restart
        assert abs(g.info.iter - s.info.iter) <= 2000 + 0.25 * s.info.iter, (p.name, g.info.iter, s.info.iter)


def test_batch_oracle_solution_parity(cuda):
    batch = problems.batch_socp_c3(count=4, seed=31, nmin=80, nmax=300)
    sols, _ = solver.rpdhg_gpu_solve_batch(batch, time_limit=300)
    for p, g in zip(batch, sols):
        o = B.solve(p, threads=2)
        assert g.info.exit_status == "optimal" and o["exit_code"] == 0
        eg = B.evaluate(p, g.primal, g.dual)
        eo = B.evaluate(p, o["x"], o["y"])
        assert_objective(p, eg["pobj"], "batch")
        assert_objective(p, eo["pobj"], "oracle")


def test_batch_infeasible_members_keep_their_status(cuda):
    batch = [problems.primal_infeasible_lp(), problems.mixed_small(seed=7), problems.dual_infeasible_lp()]
    sols, _ = solver.rpdhg_gpu_solve_batch(batch, time_limit=300)
    single = [solver.solve_problem(p, time_limit=120) for p in batch]
    cls = lambda c: {2: "p", 3: "p", 4: "d", 5: "d"}.get(c, c)
    for g, s in zip(sols, single):
        assert cls(g.info.exit_code) == cls(s.info.exit_code), (g, s)
    assert sols[1].info.exit_status == "optimal"


def test_batch_kkt_restart_variant(cuda):
    batch = _mixed_batch()[:3]
    kw = dict(time_limit=300, use_kkt_restart=True, use_duality_gap_restart=False)
    sols, _ = solver.rpdhg_gpu_solve_batch(batch, **kw)
    for p, g in zip(batch, sols):
        s = solver.solve_problem(p, **kw)
        assert g.info.exit_status == s.info.exit_status == "optimal"
        assert_objective(p, g.info.pObj, "batch")
        assert_objective(p, s.info.pObj, "single")


def test_batch_resolving_fallback_is_the_single_solve(cuda):
    batch = _mixed_batch()[:2]
    sols, info = solver.rpdhg_gpu_solve_batch(batch, time_limit=300, force_resolving=True)
    assert info.single_fallbacks == 2
    for p, g in zip(batch, sols):
        s = solver.solve_problem(p, time_limit=120, force_resolving=True)
        assert g.info.exit_code == s.info.exit_code
        assert g.info.iter == s.info.iter
        assert np.array_equal(g.primal, s.primal)


def test_batch_validation(cuda):
    ok = problems.mixed_small().kwargs()
    bad = dict(ok)
    bad["mGzero"] = ok["mGzero"] + 1
    with pytest.raises(ValueError):
        solver.rpdhg_gpu_solve_batch([ok, bad])
    extra = problems.random_feasible(n_box=5, soc_x=[3], mGnonnegative=4, density=0.5, seed=3).kwargs()
    extra["n"] += 1  # a variable outside every cone
    extra["c"] = np.append(extra["c"], 0.0)
    import scipy.sparse as sp
    extra["G"] = sp.hstack([sp.csr_matrix(extra["G"]), sp.csr_matrix((extra["m"], 1))]).tocsr()
    with pytest.raises(RuntimeError, match="status -7"):
        solver.rpdhg_gpu_solve_batch([ok, extra])


def test_batch_handle_resolves_identically(cuda):
    batch = _mixed_batch()[:3]
    with solver.BatchHandle(batch) as h:
        a, _ = h.solve(attempt_limit=50)
        b, _ = h.solve(attempt_limit=50)
        c, info = h.solve()
    one, _ = solver.rpdhg_gpu_solve_batch(batch)
    for x, y, z, w in zip(a, b, c, one):
        assert np.array_equal(x.primal, y.primal) and x.info.iter == 50  # cold start each time
        assert z.info.exit_status == w.info.exit_status == "optimal"
        assert z.info.iter == w.info.iter and np.array_equal(z.primal, w.primal)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_tiled_spmv_matches_binned(cuda, precision):
    """The instance-tiled SpMV (column segments in shared memory, 16-bit local
    columns, FP64 sums) and the binned row schedule give the same iterates up to
    summation order, and the same solutions."""
    batch = _mixed_batch() + problems.batch_socp_c3(count=12, seed=3, nmin=50, nmax=1500)
    # FP32: the binned kernel sums in FP32, the tiled one in FP64; the adaptive
    # steps amplify that difference over attempts, so FP32 compares early iterates
    attempts, tol = (60, 1e-10) if precision == "fp64" else (7, 2e-5)
    a, ia = solver.rpdhg_gpu_solve_batch(batch, attempt_limit=attempts, precision=precision)
    b, ib = solver.rpdhg_gpu_solve_batch(batch, attempt_limit=attempts, precision=precision, spmv_tiles=False)
    assert ia.spmv_tiled and not ib.spmv_tiled
    for p, g, h in zip(batch, a, b):
        for u, v in ((g.primal, h.primal), (g.dual, h.dual)):
            assert np.abs(u - v).max() <= tol * max(1.0, np.abs(v).max()), (p.name, np.abs(u - v).max())
    a, _ = solver.rpdhg_gpu_solve_batch(batch, precision=precision)
    b, _ = solver.rpdhg_gpu_solve_batch(batch, precision=precision, spmv_tiles=False)
    for p, g, h in zip(batch, a, b):
        assert g.info.exit_status == h.info.exit_status == "optimal", p.name
        assert_objective(p, g.info.pObj, "tiled")
        assert_objective(p, h.info.pObj, "binned")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_tail_kernel_solutions(cuda, precision):
    """Uneven batch whose last instances run in the tail kernel (a CTA per
    instance looping over its attempts): every instance reaches the criteria
    under the oracle's evaluator and matches its single-instance solve."""
    batch = problems.batch_socp_c3(count=48, seed=7, nmin=40, nmax=600)
    sols, info = solver.rpdhg_gpu_solve_batch(batch, precision=precision, time_limit=300)
    assert info.tail_rounds > 0, info
    for p, g in zip(batch, sols):
        assert g.info.exit_status == "optimal", (p.name, g)
        e = B.evaluate(p, g.primal, g.dual)
        assert max(e["primal_res_gpu_form"], e["dual_res"], e["rel_gap"]) < 1.05e-6, (p.name, e)
        s = solver.solve_problem(p)
        assert s.info.exit_status == "optimal", (p.name, s)
        assert_objective(p, g.info.pObj, "batch")
        assert_objective(p, s.info.pObj, "single")
