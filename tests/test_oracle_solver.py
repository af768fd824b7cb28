"""End-to-end checks of the oracle solver (CPU)."""
import numpy as np
import pytest
from scipy.optimize import linprog

from oracle import binding as B
from pdcs_b200 import problems


def test_lp_matches_highs():
    p = problems.random_feasible(n_box=60, mGzero=10, mGnonnegative=40, density=0.2, seed=3)
    mz = p.mGzero
    Gd = p.G.toarray()
    ref = linprog(p.c, A_ub=-Gd[mz:], b_ub=-p.h[mz:], A_eq=Gd[:mz], b_eq=p.h[:mz],
                  bounds=list(zip(p.bl, p.bu)), method="highs")
    assert ref.status == 0
    r = B.solve(p, threads=2)
    assert r["exit_code"] == 0
    assert abs(r["primal_objective"] - ref.fun) <= 1e-5 * (1 + abs(ref.fun))
    assert np.abs(r["x"] - ref.x).max() < 1e-4


@pytest.mark.parametrize("name", ["socp_c0", "mixed_small", "logreg_small"])
def test_oracle_converges(name):
    if name == "socp_c0":
        p = problems.socp_c0()
    elif name == "mixed_small":
        p = problems.mixed_small()
    else:
        p = problems.logreg_exp_c1(samples=200, features=20, density=0.2)
    r = B.solve(p, threads=2)
    assert r["exit_code"] == 0, r
    ev = B.evaluate(p, r["x"], r["y"])
    # the solver stops on the GPU-code criteria; the README form agrees to within rounding
    assert max(ev["primal_res_gpu_form"], ev["dual_res"], ev["rel_gap"]) < 1.05e-6
    assert ev["max_rel"] < 1e-5


def test_cpu_semantics_flag_also_converges():
    p = problems.socp_c0()
    r = B.solve(p, threads=2, cpu_semantics=1)
    assert r["exit_code"] == 0


def test_attempt_limit_stops():
    p = problems.socp_c0()
    r = B.solve(p, threads=1, attempt_limit=37)
    assert r["exit_code"] == 10 and r["iter"] == 37


def test_preconditioner_equilibrates():
    p = problems.socp_c0()
    Dr, Dl, val = B.precondition(p)
    G = p.G.tocsr().copy()
    G.data = val
    rowmax = np.abs(G).max(axis=1).toarray().ravel()
    assert np.all(np.isfinite(Dr)) and np.all(Dr > 0) and np.all(Dl > 0)
    nz = rowmax > 0
    assert np.median(rowmax[nz]) < 2.0


@pytest.mark.parametrize("name,code", [("primal_infeasible_lp", 2), ("dual_infeasible_lp", 5)])
def test_oracle_infeasibility_certificates(name, code):
    p = getattr(problems, name)()
    r = B.solve(p, threads=1, time_limit=60)
    assert r["exit_code"] == code
