"""Generate tests/golden/c2_oracle.json: the oracle's solve of the full-size
robust-portfolio workload (pdcs_b200.problems.portfolio_c2(): 1e6 assets in
[0, 1], 200 factors at 25 % density, 1e5 SOC tracking blocks of dimension 11,
one RSOC risk block of 1 000 202 elements, a budget row; 5.3e7 nonzeros).  The
oracle needs hours of CPU for it, so the GPU solves of the same seeded
instance are compared with this frozen record: the oracle's solve at 1e-8
(attempts, objective, the shared evaluator's criteria at its point, CPU seconds
per attempt) and checksums of the instance's data, which the comparison
recomputes to make sure it solves the same instance.
Run:  python tests/golden/make_c2_golden.py [threads]   (threads 0: all cores)
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import binding as B  # noqa: E402
from pdcs_b200 import problems  # noqa: E402


def checksums(p):
    G = p.G.tocsr()
    return {"n": p.n, "m": p.m, "nnz": int(G.nnz), "sum_G": float(np.sum(G.data)),
            "sum_abs_G": float(np.sum(np.abs(G.data))), "sum_c": float(np.sum(p.c)), "sum_h": float(np.sum(p.h))}


def make(threads=0):
    p = problems.portfolio_c2()
    t = time.time()
    opt = B.solve(p, threads=threads, rel_tol=1e-8, abs_tol=1e-8, time_limit=6 * 3600.0)
    wall = time.time() - t
    e = B.evaluate(p, opt["x"], opt["y"])
    return {"instance": "problems.portfolio_c2() (n = 1e6, 200 factors at 25 %, 1e5 SOC blocks of dim 11, "
                        "RSOC risk block, seed 20261205)",
            "checksums": checksums(p),
            "optimum": {"rel_tol": 1e-8, "exit_code": opt["exit_code"], "iter": opt["iter"],
                        "primal_objective": opt["primal_objective"], "dual_objective": opt["dual_objective"],
                        "evaluator": e},
            "cpu": {"threads": threads if threads > 0 else os.cpu_count(), "wall_s": wall,
                    "solve_s": opt["solve_seconds"], "setup_s": opt["setup_seconds"],
                    "s_per_attempt": opt["solve_seconds"] / max(1, opt["iter"])}}


if __name__ == "__main__":
    d = make(int(sys.argv[1]) if len(sys.argv) > 1 else 0)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c2_oracle.json")
    json.dump(d, open(path, "w"), indent=1)
    print(json.dumps(d, indent=1))
