"""The exponential-cone workload at full size (l1-logistic regression in
exp-cone form, 20000 x 500 at 5 % density: n = 61000, m = 140000, 1.12 M
nonzeros, 40000 exponential cones), plain FP64 and FP32 bulk, against the
oracle's solve of the same seeded instance frozen in tests/golden/c1_oracle.json
(tests/golden/make_c1_golden.py; the oracle needs minutes of CPU here): both
GPU solutions meet the 1e-6 criteria under the oracle's FP64 evaluator and
their objectives lie within 1e-6 of the optimum (the oracle at 1e-8)."""
import json
import os

import numpy as np
import pytest

from oracle import binding as B
from pdcs_b200 import problems, solver

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c1_oracle.json")


@pytest.fixture(scope="module")
def c1():
    g = json.load(open(GOLDEN))
    p = problems.logreg_exp_c1()
    G = p.G.tocsr()
    cs = g["checksums"]
    assert (p.n, p.m, G.nnz) == (cs["n"], cs["m"], cs["nnz"])
    for key, val in (("sum_G", np.sum(G.data)), ("sum_abs_G", np.sum(np.abs(G.data))), ("sum_c", np.sum(p.c)),
                     ("sum_h", np.sum(p.h))):
        assert abs(val - cs[key]) <= 1e-12 * max(1.0, abs(cs[key])), key  # the fixture's instance
    return p, g


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_c1_full_size_matches_oracle(cuda, c1, precision):
    p, g = c1
    s = solver.solve_problem(p, precision=precision, time_limit=300)
    assert s.info.exit_status == "optimal", s
    e = B.evaluate(p, s.primal, s.dual)
    assert max(e["primal_res_gpu_form"], e["dual_res"], e["rel_gap"]) < 1.05e-6, e
    opt = g["optimum"]["primal_objective"]
    err = abs(e["pobj"] - opt) / (1.0 + abs(opt))
    print(f"c1 {precision}: {s.info.iter} attempts (oracle {g['oracle_1e-6']['iter']}), objective error vs the "
          f"optimum {err:.2e}, criteria {e['primal_res_gpu_form']:.2e} {e['dual_res']:.2e} {e['rel_gap']:.2e}")
    assert err <= 1e-6, (e["pobj"], opt)
