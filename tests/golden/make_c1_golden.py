"""Generate tests/golden/c1_oracle.json: the oracle's solve of the full-size
exponential-cone workload (l1-logistic regression, 20000 x 500 at 5 %,
pdcs_b200.problems.logreg_exp_c1()) -- too slow to repeat inside the GPU
tests (minutes of CPU) -- so the GPU solve of the same seeded instance can be
compared with it: the optimum (oracle at 1e-8), the oracle's 1e-6 solution
(attempts, objective, criteria under the shared evaluator) and checksums of
the instance's data, which the test recomputes to make sure it solves the
same instance.
Run:  python tests/golden/make_c1_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import binding as B  # noqa: E402
from pdcs_b200 import problems  # noqa: E402


def checksums(p):
    G = p.G.tocsr()
    return {"n": p.n, "m": p.m, "nnz": int(G.nnz), "sum_G": float(np.sum(G.data)),
            "sum_abs_G": float(np.sum(np.abs(G.data))), "sum_c": float(np.sum(p.c)), "sum_h": float(np.sum(p.h))}


def make():
    p = problems.logreg_exp_c1()
    opt = B.solve(p, threads=0, rel_tol=1e-8, abs_tol=1e-8)
    o = B.solve(p, threads=0)
    e = B.evaluate(p, o["x"], o["y"])
    return {"instance": "problems.logreg_exp_c1() (20000 x 500, 5 % density, lambda 0.01, seed 20261204)",
            "checksums": checksums(p),
            "optimum": {"rel_tol": 1e-8, "exit_code": opt["exit_code"], "iter": opt["iter"],
                        "primal_objective": opt["primal_objective"]},
            "oracle_1e-6": {"exit_code": o["exit_code"], "iter": o["iter"], "primal_objective": o["primal_objective"],
                            "evaluator": e}}


if __name__ == "__main__":
    d = make()
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c1_oracle.json")
    json.dump(d, open(path, "w"), indent=1)
    print(json.dumps(d, indent=1))
