"""Bounded solve runner for profiling:  python -m pdcs_b200.profile --workload logreg --attempts 64
(or --workload batch --count 4096 --precision fp32: the batched uneven-SOCP workload;
--workload portfolio --assets 1000000: the robust portfolio with its huge risk cone)

Builds a seeded workload, uploads it to the GPU and runs the solver for a fixed
number of PDHG attempts (or to convergence with --attempts 0), printing the
result.  Used for the ncu launch lists and captures under profiles/.
"""
import argparse
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="logreg", choices=["logreg", "logreg_small", "socp", "mixed", "batch",
                                                                 "portfolio"])
    ap.add_argument("--count", type=int, default=4096, help="instances of the batch workload")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--attempts", type=int, default=64)
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--features", type=int, default=500)
    ap.add_argument("--assets", type=int, default=1_000_000)
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args(argv)
    import numpy as np
    import torch
    from . import problems, solver
    if a.workload == "batch":
        batch = problems.batch_socp_c3(count=a.count)
        with solver.BatchHandle(batch, precision=a.precision) as h:
            for _ in range(a.repeat):
                sols, info = h.solve(attempt_limit=a.attempts)
        print(f"batch of {a.count}: iter max {max(s.info.iter for s in sols)}", info, file=sys.stderr)
        return 0
    if a.workload == "logreg":
        p = problems.logreg_exp_c1(samples=a.samples, features=a.features)
    elif a.workload == "logreg_small":
        p = problems.logreg_exp_c1(samples=2000, features=100)
    elif a.workload == "portfolio":
        p = problems.portfolio_c2(n=a.assets)
    elif a.workload == "socp":
        p = problems.socp_c0()
    else:
        p = problems.mixed_small(scale=20)
    dev = torch.device("cuda", 0)
    G = p.G.tocsr()
    t = lambda x, dt=torch.float64: torch.as_tensor(np.asarray(x), dtype=dt, device=dev)
    kw = p.kwargs()
    kw.update(c=t(p.c), h=t(p.h), bl=t(p.bl), bu=t(p.bu),
              G=(t(G.indptr, torch.int32), t(G.indices, torch.int32), t(G.data)))
    for _ in range(a.repeat):
        sol = solver.rpdhg_gpu_solve(**kw, attempt_limit=a.attempts, precision=a.precision)
    print(sol, "kernels", sol.info.kernel_launches, file=sys.stderr)
    return 0


if __name__ == "__main__":
    sys.exit(main())
