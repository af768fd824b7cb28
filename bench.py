#!/usr/bin/env python
"""Benchmark: time-to-1e-6 KKT and PDHG iterations/s on the exponential-cone
logistic-regression program (20000 samples x 500 features, 5% density, FP64).

A step is one complete solve from a cold start to the reference's 1e-6
relative criteria.  `value` is PDHG iterations per second over the timed
steps with the problem already resident in HBM; `e2e` is the same metric
through the public Python API from host numpy buffers (host->device copy of
the problem and device->host copy of the solution inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one process per GPU, weak scaling); the
path has no collective.  `--impl reference` times the CPU restatement of the
reference (the reference itself is Julia + CUDA.jl and cannot run here) on
the host cores, on bounded samples of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-1e-6 KKT & iter/s: batched mixed-prec vs plain FP64 PDHG, 1 B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--features", type=int, default=500)
    ap.add_argument("--cpu-attempts", type=int, default=300,
                    help="PDHG attempts per bounded CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def workload(args):
    from pdcs_b200 import problems
    p = problems.logreg_exp_c1(samples=args.samples, features=args.features)
    cfg = {"workload": f"l1-logistic regression in exp-cone form, {args.samples}x{args.features} "
                       f"@5% (n={p.n}, m={p.m}, nnz={p.nnz}, {p.expG} exp cones)",
           "n": p.n, "m": p.m, "nnz": p.nnz, "seed": p.seed, "tolerance": 1e-6,
           "l2": "256 MiB buffer written between timed steps (problem fits in L2 within a solve)"}
    return p, cfg


def bytes_per_iter(p, w=8):
    """Algorithmic HBM bytes of one PDHG iteration: G and G' (values + int32
    column indices) once each, both row pointers, the primal/dual vector
    streams, the box bounds and the averaged iterates."""
    n, m, nnz, n1 = p.n, p.m, p.nnz, p.nb
    return 2 * nnz * (w + 4) + 4 * (m + 1) + 4 * (n + 1) + w * (4 * n + 2 * n1 + 4 * m) + w * 2 * (n + m)


class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, flags in rows for i, f in enumerate(flags) if f.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(p, attempts):
    """The oracle (CPU restatement) on all host cores, bounded sample."""
    from oracle import binding as B
    cores = os.cpu_count() or 1
    r = B.solve(p, threads=cores, attempt_limit=attempts)
    secs = r["solve_seconds"]
    return {"value": r["iter"] / secs, "unit": "iter/s", "cores": cores, "kind": "port",
            "sample": f"first {r['iter']} PDHG attempts of one solve of the same instance "
                      f"({secs:.1f} s of CPU time, setup excluded)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    p, cfg = workload(args)
    from oracle import binding as B
    cores = os.cpu_count() or 1
    for _ in range(max(0, min(args.warmup, 1))):
        B.solve(p, threads=cores, attempt_limit=20)
    iters, secs = 0, 0.0
    for _ in range(args.steps):
        r = B.solve(p, threads=cores, attempt_limit=args.cpu_attempts)
        iters += r["iter"]
        secs += r["solve_seconds"]
    v = iters / secs
    line = {"metric": METRIC, "impl": "reference", "value": v, "unit": "iter/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": cfg,
            "cpu_baseline": {"value": v, "unit": "iter/s", "cores": cores, "kind": "port",
                             "sample": f"each step: first {args.cpu_attempts} PDHG attempts of a solve "
                                       "(the reference's Julia/CUDA.jl code cannot run here; this is the "
                                       "C++ restatement of its algorithm)"},
            "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def device_problem(p, dev):
    import numpy as np
    import torch
    G = p.G.tocsr()
    t = lambda a, dt=torch.float64: torch.as_tensor(np.asarray(a), dtype=dt, device=dev)
    kw = p.kwargs()
    kw.update(c=t(p.c), h=t(p.h), bl=t(p.bl), bu=t(p.bu),
              G=(t(G.indptr, torch.int32), t(G.indices, torch.int32), t(G.data)))
    return kw


def timed_solve(kw, stream, **extra):
    import torch
    from pdcs_b200 import solver
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    sol = solver.rpdhg_gpu_solve(**kw, stream=stream.cuda_stream, **extra)
    e.record(stream)
    e.synchronize()
    return sol, s.elapsed_time(e) * 1e-3


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    p, cfg = workload(args)
    kw_dev = device_problem(p, dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        sol, _ = timed_solve(kw_dev, stream)
    assert sol.info.exit_status == "optimal", sol

    # ---- device-resident timed region ----
    total_t, total_it, launches, sols = 0.0, 0, 0, []
    barrier()
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            sol, t = timed_solve(kw_dev, stream)
            total_t += t
            total_it += sol.info.iter
            launches += sol.info.kernel_launches
            sols.append(sol)
    barrier()
    clocks = clk.summary()
    t_max = total_t
    it_sum = total_it
    if world > 1:
        tt = torch.tensor([total_t], dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt[0])
        ii = torch.tensor([float(total_it)], dtype=torch.float64)
        dist.all_reduce(ii, op=dist.ReduceOp.SUM)
        it_sum = int(ii[0])
    value = it_sum / t_max
    last = sols[-1].info

    # ---- per-attempt time from two bounded runs (no checkpoints below 2000 attempts) ----
    a1, a2 = 200, 1800
    _, t1 = timed_solve(kw_dev, stream, attempt_limit=a1)
    _, t2 = timed_solve(kw_dev, stream, attempt_limit=a2)
    t_att = (t2 - t1) / (a2 - a1)
    B_it = bytes_per_iter(p)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = B_it / t_att / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_logreg_c1.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get("dram_bytes_per_attempt")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": "one PDHG attempt (G'y SpMV, primal update+projection, Gx/Gx_lag SpMV, "
                          "dual update+exp-cone projection, control, reflection)",
                "algorithmic_bytes_per_attempt": B_it, "attempt_ms": t_att * 1e3,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback"}

    # ---- end to end through the public API from host buffers ----
    e2e = None
    if not args.no_e2e:
        from pdcs_b200 import solver
        kw_host = p.kwargs()
        G = p.G.tocsr()
        h2d = G.indptr.size * 4 + G.indices.size * 4 + G.data.nbytes + p.c.nbytes + p.h.nbytes + \
            p.bl.nbytes + p.bu.nbytes
        d2h = 8 * (p.n + p.m)
        et, eit = 0.0, 0
        barrier()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            sol_h = solver.rpdhg_gpu_solve(**kw_host, stream=stream.cuda_stream)
            e.record(stream)
            e.synchronize()
            et += s.elapsed_time(e) * 1e-3
            eit += sol_h.info.iter
        barrier()
        if world > 1:
            tt = torch.tensor([et], dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            et = float(tt[0])
            ii = torch.tensor([float(eit)], dtype=torch.float64)
            dist.all_reduce(ii, op=dist.ReduceOp.SUM)
            eit = int(ii[0])
        e2e = {"value": eit / et, "unit": "iter/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": 1e3 * et / args.steps, "iterations_per_solve": sol_h.info.iter}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(p, args.cpu_attempts)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": {**cfg, "parallelism": f"{world} independent replicas" if world > 1 else "single GPU"},
                "time_to_1e-6_ms": 1e3 * t_max / args.steps,
                "iterations_per_solve": last.iter, "restarts": last.restart_used,
                "kkt": {"l_inf_rel_primal_res": last.l_inf_rel_primal_res,
                        "l_inf_rel_dual_res": last.l_inf_rel_dual_res, "rel_gap": last.rel_gap},
                "setup_ms": last.setup_time * 1e3,
                "breakdown_ms": {"iterations": last.time_iterations * 1e3, "exit_checks": last.time_exit_checks * 1e3,
                                 "restarts": last.time_restarts * 1e3, "restart_probes": last.restart_probes},
                "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
                "roofline": roofline, "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
