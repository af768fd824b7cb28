"""Objective parity at the north star's bar (test helper).

A solve stopped at the 1e-6 criteria is compared with the problem's optimum,
taken from the oracle run to 1e-9 on the same instance: every reported
objective must lie within 1e-6 (relative, 1 + |optimum|) of it.  Two 1e-6
solutions can differ from each other by up to twice that, so solutions are
never compared with each other at 1e-6, only each with the optimum."""
from oracle import binding as B

OBJ_TOL = 1e-6
_cache = {}


def optimum(p):
    key = id(p)
    if key not in _cache:
        o = B.solve(p, threads=0, rel_tol=1e-9, abs_tol=1e-9, time_limit=600)
        assert o["exit_code"] == 0, (getattr(p, "name", p), o["exit_code"])
        _cache[key] = (p, o["primal_objective"])  # keep p alive so its id stays unique
    return _cache[key][1]


def objective_error(p, pobj):
    ref = optimum(p)
    return abs(pobj - ref) / (1.0 + abs(ref))


def assert_objective(p, pobj, what=""):
    err = objective_error(p, pobj)
    assert err <= OBJ_TOL, (getattr(p, "name", ""), what, pobj, optimum(p), err)
