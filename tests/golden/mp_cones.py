"""60-digit projections onto the scaled cones (fixture generation only).

Used by make_ref_golden.py to decide, block by block, which of the
reference's and the oracle's outputs is the projection where the two differ.
Every projection is computed from its KKT conditions in mpmath arithmetic:

  S o SOC  = {(t, x): t >= ||D x||}, D_i = S0/S_i:  outside the cone and its
             polar, p_x = x / (1 + mu D^2), p_t = t / (1 - mu) on the boundary,
             mu found by bisection (mu in (0, 1) for t > 0, (1, inf) for t < 0,
             mu = 1 and p_t = ||D p_x|| for t = 0);
  S o RSOC = {2 p q >= ||D z||^2, p, q >= 0}, D_i = sqrt(S0 S1)/S_i: the
             rotation ((p + q)/sqrt2, (p - q)/sqrt2) maps it isometrically onto
             the weighted SOC {u >= ||(w, D z)||};
  S o K_exp: the boundary point sp (dr rho, ds, dt e^rho) with
             v - w = lam (1/dr, (1 - rho)/ds, -e^{-rho}/dt), sp, lam > 0, rho
             the root of f on the interval where both multipliers are positive
             (bisection to 400 halvings on each admissible interval);
  S o K_exp^*: Moreau, v + P_{(1/S) o K_exp}(-v).
The bisections run 400 halvings (1500 for the exponential cone).
"""
import mpmath as mp
import numpy as np

mp.mp.dps = 60


def _vec(a):
    return [mp.mpf(float(x)) for x in a]


def _soc(t, x, D):
    nDx = mp.sqrt(sum((d * xi) ** 2 for d, xi in zip(D, x)))
    if nDx <= t:
        return t, x
    nxD = mp.sqrt(sum((xi / d) ** 2 for d, xi in zip(D, x)))
    if nxD <= -t:
        return mp.mpf(0), [mp.mpf(0)] * len(x)
    if t == 0:
        px = [xi / (1 + d * d) for d, xi in zip(D, x)]
        return mp.sqrt(sum((d * p) ** 2 for d, p in zip(D, px))), px

    def phi(mu):  # ||D x/(1 + mu D^2)|| |1 - mu| - |t|: decreasing on (0,1), increasing on (1,inf)
        return mp.sqrt(sum((d * xi / (1 + mu * d * d)) ** 2 for d, xi in zip(D, x))) * abs(1 - mu) - abs(t)

    if t > 0:
        lo, hi = mp.mpf(0), mp.mpf(1)
        for _ in range(400):
            mid = (lo + hi) / 2
            lo, hi = (mid, hi) if phi(mid) > 0 else (lo, mid)
    else:
        lo, hi = mp.mpf(1), mp.mpf(2)
        while phi(hi) < 0:
            hi *= 2
        for _ in range(400):
            mid = (lo + hi) / 2
            lo, hi = (mid, hi) if phi(mid) < 0 else (lo, mid)
    mu = (lo + hi) / 2
    px = [xi / (1 + mu * d * d) for d, xi in zip(D, x)]
    return mp.sqrt(sum((d * p) ** 2 for d, p in zip(D, px))), px


def proj_soc(v, S):
    v, S = _vec(v), _vec(S)
    D = [S[0] / s for s in S[1:]]
    t, x = _soc(v[0], v[1:], D)
    return np.array([float(t)] + [float(a) for a in x])


def proj_rsoc(v, S):
    v, S = _vec(v), _vec(S)
    D = [mp.sqrt(S[0] * S[1]) / s for s in S[2:]]
    r2 = mp.sqrt(2)
    u, w = (v[0] + v[1]) / r2, (v[0] - v[1]) / r2
    t, x = _soc(u, [w] + v[2:], [mp.mpf(1)] + D)
    p, q = (t + x[0]) / r2, (t - x[0]) / r2
    return np.array([float(p), float(q)] + [float(a) for a in x[1:]])


def _exp(v, D):
    r, s, t = v
    dr, ds, dt = D
    rr, ss, tt = r / dr, s / ds, t / dt
    if (ss > 0 and ss * mp.e ** (rr / ss) <= tt) or (ss == 0 and rr <= 0 and tt >= 0):
        return [r, s, t]
    a, b, c = -dr * r, -ds * s, -dt * t
    if (a < 0 and -a * mp.e ** (b / a) <= mp.e * c) or (a == 0 and b >= 0 and c >= 0):
        return [mp.mpf(0)] * 3
    if r <= 0 and s <= 0:
        return [r, mp.mpf(0), max(t, mp.mpf(0))]

    def Q(x):
        return ds * ds + dr * dr * x * (x - 1)

    def N1(x):
        return dr * r * (x - 1) + ds * s

    def N2(x):
        return ds * r - dr * s * x

    def f(x):
        return N1(x) * dt * mp.e ** x - dr * ds * N2(x) * mp.e ** (-x) / dt - t * Q(x)

    bps = []
    if r != 0:
        bps.append(1 - ds * s / (dr * r))
    if s != 0:
        bps.append(ds * r / (dr * s))
    disc = 1 - 4 * (ds / dr) ** 2
    if disc >= 0:
        bps += [(1 - mp.sqrt(disc)) / 2, (1 + mp.sqrt(disc)) / 2]
    edges = [None] + sorted(bps) + [None]
    for k in range(len(edges) - 1):
        lo, hi = edges[k], edges[k + 1]
        if lo is None and hi is None:
            p = mp.mpf(0)
        elif lo is None:
            p = hi - 1
        elif hi is None:
            p = lo + 1
        else:
            p = (lo + hi) / 2
        q = Q(p)
        if not (N1(p) * q > 0 and N2(p) * q > 0):
            continue
        sg = 1 if q > 0 else -1
        if lo is None:
            lo = p - 1
            while sg * f(lo) >= 0:
                lo = p - 2 * (p - lo)
        if hi is None:
            hi = p + 1
            while sg * f(hi) <= 0:
                hi = p + 2 * (hi - p)
        neg_lo = sg * f(lo) < 0
        for _ in range(1500):
            mid = (lo + hi) / 2
            lo, hi = (mid, hi) if (sg * f(mid) < 0) == neg_lo else (lo, mid)
        rho = (lo + hi) / 2
        sp = N1(rho) / Q(rho)
        return [sp * dr * rho, sp * ds, sp * dt * mp.e ** rho]
    raise RuntimeError("no admissible root")


# Near a root of N1 the root sits e^{-|rho|}-close to it (|rho| up to a few
# hundred here), so the exponential cone runs at 400 digits.
def proj_exp(v, S):
    with mp.workdps(400):
        return np.array([float(a) for a in _exp(_vec(v), _vec(S))])


def proj_dexp(v, S):
    with mp.workdps(400):
        v, S = _vec(v), _vec(S)
        w = _exp([-a for a in v], [1 / s for s in S])
        return np.array([float(a + b) for a, b in zip(v, w)])


PROJ = {"soc": proj_soc, "rsoc": proj_rsoc, "exp": proj_exp, "dexp": proj_dexp}
