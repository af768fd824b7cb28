"""End-to-end parity of the CUDA solver against the oracle (same seeded inputs)."""
import numpy as np
import pytest

from oracle import binding as B
from _parity import assert_objective
from pdcs_b200 import problems, solver

pytestmark = pytest.mark.gpu

INSTANCES = {
    "socp_c0": lambda: problems.socp_c0(),
    "mixed_small": lambda: problems.mixed_small(),
    "mixed_medium": lambda: problems.mixed_small(seed=9, scale=6),
    "logreg_small": lambda: problems.logreg_exp_c1(samples=300, features=30, density=0.2),
}


@pytest.mark.parametrize("name", ["socp_c0", "mixed_small", "logreg_small"])
@pytest.mark.parametrize("attempts", [1, 7, 60])
def test_first_attempts_track_oracle(cuda, name, attempts):
    """Same algorithm, same data: the first iterates agree to rounding."""
    p = INSTANCES[name]()
    g = solver.solve_problem(p, attempt_limit=attempts)
    o = B.solve(p, threads=1, attempt_limit=attempts)
    assert g.info.exit_code == 10 and o["exit_code"] == 10
    assert g.info.iter == o["iter"] == attempts
    for a, b in ((g.primal, o["x"]), (g.dual, o["y"])):
        scale = max(1.0, np.abs(b).max())
        assert np.abs(a - b).max() <= 1e-9 * scale, (name, attempts, np.abs(a - b).max())


@pytest.mark.parametrize("name", list(INSTANCES))
def test_solution_parity(cuda, name):
    p = INSTANCES[name]()
    g = solver.solve_problem(p, time_limit=120)
    o = B.solve(p, threads=4)
    assert g.info.exit_status == "optimal", g
    assert o["exit_code"] == 0
    eg = B.evaluate(p, g.primal, g.dual)
    eo = B.evaluate(p, o["x"], o["y"])
    # tolerance 1e-6 on the criteria the solver stops on (GPU-code denominators),
    # with a small allowance for the evaluator's own rounding
    for e in (eg, eo):
        assert max(e["primal_res_gpu_form"], e["dual_res"], e["rel_gap"]) < 1.05e-6, e
    assert_objective(p, eg["pobj"], "gpu")
    assert_objective(p, eo["pobj"], "oracle")
    assert abs(g.info.pObj - eg["pobj"]) <= 1e-9 * (1 + abs(eg["pobj"]))


def test_device_resident_inputs(cuda):
    import torch
    p = problems.mixed_small()
    G = p.G.tocsr()
    t = lambda a, dt=torch.float64: torch.as_tensor(np.asarray(a), dtype=dt, device=cuda)
    kw = p.kwargs()
    kw.update(c=t(p.c), h=t(p.h), bl=t(p.bl), bu=t(p.bu),
              G=(t(G.indptr, torch.int32), t(G.indices, torch.int32), t(G.data)))
    g = solver.rpdhg_gpu_solve(**kw, device_output=True, time_limit=120)
    h = solver.solve_problem(p, time_limit=120)
    assert g.info.exit_status == "optimal"
    assert np.allclose(g.primal.cpu().numpy(), h.primal, atol=1e-12)


def test_warm_start_matches_oracle(cuda):
    p = problems.socp_c0()
    first = solver.solve_problem(p, time_limit=120)
    again = solver.solve_problem(p, time_limit=120, warm_start=True, primal_sol=first.primal, dual_sol=first.dual)
    o = B.solve(p, threads=2, warm_x=first.primal, warm_y=first.dual)
    assert again.info.exit_status == "optimal" and o["exit_code"] == 0
    assert again.info.iter == o["iter"]
    w = solver.solve_problem(p, attempt_limit=30, warm_start=True, primal_sol=first.primal, dual_sol=first.dual)
    ow = B.solve(p, threads=1, attempt_limit=30, warm_x=first.primal, warm_y=first.dual)
    assert np.abs(w.primal - ow["x"]).max() <= 1e-9 * max(1.0, np.abs(ow["x"]).max())


def test_kkt_restart_variant(cuda):
    p = problems.mixed_small()
    g = solver.solve_problem(p, time_limit=120, use_kkt_restart=True, use_duality_gap_restart=False)
    o = B.solve(p, threads=2, use_kkt_restart=1, use_duality_gap_restart=0)
    assert g.info.exit_status == "optimal" and o["exit_code"] == 0
    assert_objective(p, g.info.pObj, "gpu")
    assert_objective(p, o["primal_objective"], "oracle")


@pytest.mark.parametrize("name", ["primal_infeasible_lp", "dual_infeasible_lp"])
def test_infeasibility_status_matches_oracle(cuda, name):
    p = getattr(problems, name)()
    g = solver.solve_problem(p, time_limit=60)
    o = B.solve(p, threads=1, time_limit=60)
    # same certificate class (primal: 2/3, dual: 4/5); the low/high accuracy
    # label depends on objective trends that differ with rounding
    cls = {2: "primal", 3: "primal", 4: "dual", 5: "dual"}
    assert cls.get(g.info.exit_code) == cls.get(o["exit_code"]) is not None, (g.info.exit_code, o["exit_code"])


@pytest.mark.parametrize("name", ["socp_c0", "mixed_small"])
def test_resolving_fallback_matches_oracle(cuda, name):
    """resolving_pessimistic_step!: power-method step, fixed-step PDHG, uniform averaging."""
    p = INSTANCES[name]()
    g = solver.solve_problem(p, force_resolving=True, attempt_limit=40)
    o = B.solve(p, threads=1, force_resolving=1, attempt_limit=40)
    assert g.info.iter == o["iter"] == 40
    assert np.abs(g.primal - o["x"]).max() <= 1e-9 * max(1.0, np.abs(o["x"]).max())
    g = solver.solve_problem(p, force_resolving=True, time_limit=120)
    o = B.solve(p, threads=2, force_resolving=1, time_limit=120)
    assert g.info.exit_status == "optimal" and o["exit_code"] == 0
    assert_objective(p, g.info.pObj, "gpu")
    assert_objective(p, o["primal_objective"], "oracle")


def test_spmv_schedules_agree(cuda):
    """Every SpMV schedule (nonzeros per lane: 1 lane per row up to a CTA per row) gives the
    same iterates to rounding; the autotuned default reports the schedule it picked."""
    p = problems.logreg_exp_c1(samples=400, features=40, density=0.2)
    ref = solver.solve_problem(p, attempt_limit=20, spmv_lane_nnz=4)
    assert ref.info.spmv_lane_nnz == (4, 4)
    for lane in (0, 1, 2, 8, 16):
        g = solver.solve_problem(p, attempt_limit=20, spmv_lane_nnz=lane)
        if lane:
            assert g.info.spmv_lane_nnz == (lane, lane)
        else:  # below 2^20 nonzeros the autotuner keeps the default
            assert g.info.spmv_lane_nnz == (4, 4)
        scale = max(1.0, np.abs(ref.primal).max())
        assert np.abs(g.primal - ref.primal).max() <= 1e-9 * scale, lane
