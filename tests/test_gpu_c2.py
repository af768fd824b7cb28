"""Robust portfolio with a huge risk cone (problems.portfolio_c2, the c2
structure at n = 20000: one RSOC block of 20022 elements, 2000 SOC tracking
blocks of dim 11, a budget row).  The RSOC block is above the huge-block size,
so every projection onto it runs as part D of the update kernels (a group of
CTAs meeting at bounded barriers between the reductions of its Newton solve).
Parity with the oracle: the first attempts agree to 1e-9 (FP64), and full
solves (FP64 and FP32 bulk) meet the 1e-6 criteria under the oracle's FP64
evaluator with objectives within 1e-6 of the optimum."""
import numpy as np
import pytest

from oracle import binding as B
from _parity import assert_objective
from pdcs_b200 import problems, solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2_small():
    return problems.portfolio_c2(n=20000, factors=20)


@pytest.mark.parametrize("attempts", [1, 7, 60])
def test_c2_first_attempts_track_oracle(cuda, c2_small, attempts):
    p = c2_small
    g = solver.solve_problem(p, attempt_limit=attempts)
    o = B.solve(p, threads=1, attempt_limit=attempts)
    assert g.info.iter == o["iter"] == attempts
    for a, b in ((g.primal, o["x"]), (g.dual, o["y"])):
        err = np.abs(a - b).max() / max(1.0, np.abs(b).max())
        assert err <= 1e-9, (attempts, err)


@pytest.fixture(scope="module")
def c2_long_rows():
    """Factor rows of 35000 nonzeros and a budget row of 70000: both above the
    split-row threshold of the binned SpMV (16384), so G x runs as chunks of
    4096 nonzeros whose partials the row's last chunk adds."""
    return problems.portfolio_c2(n=70000, factors=8, load_density=0.5)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("attempts", [1, 7])
def test_c2_split_rows_track_oracle(cuda, c2_long_rows, precision, attempts):
    p = c2_long_rows
    g = solver.solve_problem(p, precision=precision, attempt_limit=attempts)
    o = B.solve(p, threads=1, attempt_limit=attempts)
    assert g.info.iter == o["iter"] == attempts
    tol = 1e-9 if precision == "fp64" else 1e-6
    for a, b in ((g.primal, o["x"]), (g.dual, o["y"])):
        err = np.abs(a - b).max() / max(1.0, np.abs(b).max())
        assert err <= tol, (attempts, err)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_c2_solution_meets_criteria(cuda, c2_small, precision):
    p = c2_small
    g = solver.solve_problem(p, precision=precision, time_limit=300)
    assert g.info.exit_status == "optimal", g
    e = B.evaluate(p, g.primal, g.dual)
    assert max(e["primal_res_gpu_form"], e["dual_res"], e["rel_gap"]) < 1.05e-6, e
    assert_objective(p, e["pobj"], precision)
