"""Independent numpy checks of the cone projections (test helpers).

These pin the oracle's projections without trusting its algorithm: a candidate
p = P_C(v) is accepted when p lies in C and ||v - p|| is no larger than the
distance found by a brute-force global search over the boundary rays of C
(projection onto a closed convex cone is the unique minimiser, and by strong
convexity ||p - p*||^2 <= ||v - p||^2 - ||v - p*||^2).
"""
import math

import numpy as np


def _in_kexp_exact(u):
    r, s, t = u
    if s > 0:
        if t <= 0:
            return False
        return math.log(s) + r / s <= math.log(t)  # s exp(r/s) <= t without overflow
    return r <= 0 and s == 0 and t >= 0


def in_scaled_exp(p, D, tol=1e-9):
    """p lies within distance ~tol*max(1, ||p||) of D o K_exp (K_exp =
    cl{(r, s, t): s > 0, s exp(r / s) <= t}): the point nudged by eps
    towards the cone's interior direction (-1, 0, +1) is inside."""
    p = np.asarray(p, float)
    eps = tol * max(1.0, float(np.linalg.norm(p)))
    q = p + eps * np.array([-1.0, 0.0, 1.0])
    q[1] = max(q[1], 0.0) if abs(q[1]) <= eps else q[1]
    return _in_kexp_exact(q / D)


def brute_exp_distance(v, D):
    """min over w in D o K_exp of ||v - w||, by scanning boundary rays
    rho = sinh(z), z in [-12, 12], plus the two faces of the cone's closure."""
    v = np.asarray(v, float)
    best = float(np.linalg.norm(v))                       # w = 0
    face = np.array([min(v[0], 0.0), 0.0, max(v[2], 0.0)])  # {r <= 0, s = 0, t >= 0}
    best = min(best, float(np.linalg.norm(v - face)))

    def ray_dist(rho):
        rho = np.asarray(rho, float)
        with np.errstate(over="ignore", under="ignore", invalid="ignore"):
            a = np.stack([D[0] * rho, D[1] * np.ones_like(rho), D[2] * np.exp(np.minimum(rho, 700))])
            nrm = np.linalg.norm(a, axis=0)
            a = a / nrm
            proj = np.maximum(a.T @ v, 0.0)
            d2 = v @ v - proj ** 2
        return np.sqrt(np.maximum(d2, 0.0))

    z = np.linspace(-12, 12, 200001)
    rho = np.sinh(z)
    d = ray_dist(rho)
    k = int(np.nanargmin(d))
    lo, hi = z[max(k - 1, 0)], z[min(k + 1, len(z) - 1)]
    for _ in range(200):  # golden-section refinement around the best grid point
        g = (math.sqrt(5) - 1) / 2
        a1 = hi - g * (hi - lo)
        a2 = lo + g * (hi - lo)
        if ray_dist(np.sinh(a1)) < ray_dist(np.sinh(a2)):
            hi = a2
        else:
            lo = a1
    best = min(best, float(np.nanmin(d)), float(ray_dist(np.sinh(0.5 * (lo + hi)))))
    return best


def check_exp_projection(v, p, D, tol=1e-9):
    v, p, D = (np.asarray(a, float) for a in (v, p, D))
    nv = max(1.0, float(np.linalg.norm(v)))
    if not in_scaled_exp(p, D):
        return False, "infeasible"
    dp = float(np.linalg.norm(v - p))
    db = brute_exp_distance(v, D)
    if dp ** 2 > db ** 2 + tol * nv ** 2:
        return False, f"not minimal: {dp} > {db}"
    return True, ""


def soc_project_reference(v, Dw=None):
    """Weighted-SOC projection by bisection on the KKT multiplier (slow, safe)."""
    v = np.asarray(v, float)
    t, x = v[0], v[1:]
    D = np.ones_like(x) if Dw is None else np.asarray(Dw, float)
    if np.linalg.norm(D * x) <= t:
        return v.copy()
    if np.linalg.norm(x / D) <= -t:
        return np.zeros_like(v)
    # phi(mu) = ||D x/(1+mu D^2)|| - t/(1-mu), root in mu in (0,1) for t>0, (1,inf) for t<0
    def phi(mu):
        return np.linalg.norm(D * x / (1 + mu * D * D)) * abs(1 - mu) - abs(t) if t != 0 else None
    if t == 0:
        mu = 1.0
    else:
        if t > 0:
            lo, hi = 0.0, 1.0
            for _ in range(2000):
                mid = 0.5 * (lo + hi)
                if phi(mid) > 0:
                    lo = mid
                else:
                    hi = mid
        else:
            lo, hi = 1.0, 2.0
            while phi(hi) < 0:
                hi *= 2
            for _ in range(2000):
                mid = 0.5 * (lo + hi)
                if phi(mid) < 0:
                    lo = mid
                else:
                    hi = mid
        mu = 0.5 * (lo + hi)
    y = x / (1 + mu * D * D)
    s = np.linalg.norm(D * y)
    return np.concatenate([[s], y])


# ---------------------------------------------------------------------------
# KKT residual of a candidate projection p of v onto a scaled cone C = S o K
# (the sets the solver's block projections use: p / S in K).  p is the
# projection iff p in C, q = p - v in the dual cone C* = (1/S) o K*, and
# <p, q> = 0.  kkt_residual returns the largest of the three violations,
# relative to max(1, ||v||) (squared for the products), so two differing
# candidates can be ranked: the exact projection has a residual at the
# rounding level, an approximate one (a root search stopped at a tolerance, a
# wrong branch) a larger one.
# ---------------------------------------------------------------------------

def _soc_in(u, D):     # {t >= ||D x||}
    return max(0.0, float(np.linalg.norm(D * u[1:])) - u[0])


def _rsoc_in(u, D):    # {2 x y >= ||D z||^2, x, y >= 0}, as a length
    quad = float(np.sum((D * u[2:]) ** 2)) - 2.0 * u[0] * u[1]
    return max(0.0, -u[0], -u[1], quad / max(1e-300, abs(u[0]) + abs(u[1]) + float(np.linalg.norm(D * u[2:]))))


def _kexp_in(u):       # K_exp = cl{s > 0, s e^{r/s} <= t}
    r, s_, t = (float(x) for x in u)
    if s_ > 0.0:
        with np.errstate(over="ignore"):
            return max(0.0, s_ * math.exp(min(r / s_, 700.0)) - t)
    return max(0.0, r, -t, -s_)


def _kexp_dual_in(u):  # K_exp^* = cl{a < 0, -a e^{b/a} <= e c}
    a, b, c = (float(x) for x in u)
    if a < 0.0:
        return max(0.0, -a * math.exp(min(b / a, 700.0)) - math.e * c)
    return max(0.0, a, -b, -c)


def kkt_residual(kind, v, p, S=None):
    v = np.asarray(v, float)
    p = np.asarray(p, float)
    if not np.all(np.isfinite(p)):
        return math.inf
    d = v.size
    S = np.ones(d) if S is None else np.asarray(S, float)
    q = p - v
    sc = max(1.0, float(np.linalg.norm(v)))
    if kind == "soc":
        D = S[0] / S[1:]
        prim, dual = _soc_in(p, D), _soc_in(q, 1.0 / D)
    elif kind == "rsoc":
        D = math.sqrt(S[0] * S[1]) / S[2:]
        prim, dual = _rsoc_in(p, D), _rsoc_in(q, 1.0 / D)
    elif kind == "exp":
        prim, dual = _kexp_in(p / S), _kexp_dual_in(q * S)
    elif kind == "dexp":  # C = S o K*, C* = (1/S) o K
        prim, dual = _kexp_dual_in(p / S), _kexp_in(q * S)
    else:
        raise ValueError(kind)
    return max(prim / sc, dual / sc, abs(float(p @ q)) / sc ** 2)


def better_projection(kind, v, S, p_good, p_other, floor=1e-13):
    """p_good is the valid projection where p_other differs: p_good's KKT
    residual is at the rounding floor or no larger than p_other's."""
    rg = kkt_residual(kind, v, p_good, S)
    return rg <= floor or rg <= kkt_residual(kind, v, p_other, S)
