"""Seeded synthetic conic programs in PDCS's problem form.

    min c'x  s.t.  Gx - h in K_d,  bl <= x[:nb] <= bu,  x[nb:] in K_p

The field names follow the keyword arguments of ``rpdhg_gpu_solve``
(src/pdcs_gpu/rpdhg_alg_gpu_gen.jl:1219-1268).  All instances are feasible and
bounded by construction in the manner of the reference's example scripts
(test/test_soc.jl:8-26, test/test_exp.jl:8-28): an interior primal point x0,
an interior slack s0 in K_d and an interior dual pair (y0, lam0) are drawn and
h = G x0 - s0, c = G' y0 + lam0.

Exponential cone convention (as in the reference): K_exp = cl{(r, s, t) :
s > 0, s exp(r / s) <= t}; its dual is K_exp^* = cl{(a, b, c) : a < 0,
-a exp(b / a) <= e c}.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np
import scipy.sparse as sp


@dataclasses.dataclass
class ConicProblem:
    n: int
    m: int
    nb: int
    c: np.ndarray
    G: sp.csr_matrix
    h: np.ndarray
    mGzero: int = 0
    mGnonnegative: int = 0
    socG: List[int] = dataclasses.field(default_factory=list)
    rsocG: List[int] = dataclasses.field(default_factory=list)
    expG: int = 0
    dual_expG: int = 0
    bl: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    bu: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    soc_x: List[int] = dataclasses.field(default_factory=list)
    rsoc_x: List[int] = dataclasses.field(default_factory=list)
    exp_x: int = 0
    dual_exp_x: int = 0
    name: str = ""
    seed: int = 0

    @property
    def nnz(self) -> int:
        return int(self.G.nnz)

    def kwargs(self) -> dict:
        """Keyword arguments in the order and naming of rpdhg_gpu_solve."""
        return dict(n=self.n, m=self.m, nb=self.nb, c=self.c, G=self.G, h=self.h,
                    mGzero=self.mGzero, mGnonnegative=self.mGnonnegative,
                    socG=list(self.socG), rsocG=list(self.rsocG), expG=self.expG,
                    dual_expG=self.dual_expG, bl=self.bl, bu=self.bu,
                    soc_x=list(self.soc_x), rsoc_x=list(self.rsoc_x),
                    exp_x=self.exp_x, dual_exp_x=self.dual_exp_x)


# --------------------------------------------------------------------------
# interior points of the cones
# --------------------------------------------------------------------------

def _soc_interior(rng, d):
    v = rng.standard_normal(d - 1)
    return np.concatenate([[np.linalg.norm(v) + rng.uniform(0.5, 1.5)], v])


def _rsoc_interior(rng, d):
    z = rng.standard_normal(d - 2)
    p = rng.uniform(0.5, 2.0)
    q = (z @ z) / (2 * p) + rng.uniform(0.5, 1.5)
    return np.concatenate([[p, q], z])


def _exp_interior(rng):
    r = rng.uniform(-1.0, 1.0)
    s = rng.uniform(0.5, 1.5)
    t = s * math.exp(r / s) + rng.uniform(0.5, 1.5)
    return np.array([r, s, t])


def _dexp_interior(rng):
    a = -rng.uniform(0.5, 1.5)
    b = rng.uniform(-1.0, 1.0)
    c = -a * math.exp(b / a) / math.e + rng.uniform(0.5, 1.5)
    return np.array([a, b, c])


def _random_dims(rng, total, lo, hi):
    dims = []
    left = total
    while left > 0:
        d = int(rng.integers(lo, hi + 1))
        if left - d < lo and left - d != 0:
            d = left
        d = min(d, left)
        dims.append(d)
        left -= d
    return dims


def random_feasible(*, n_box=0, soc_x=(), rsoc_x=(), exp_x=0, dual_exp_x=0,
                    mGzero=0, mGnonnegative=0, socG=(), rsocG=(), expG=0, dual_expG=0,
                    density=0.01, seed=0, box=(-10.0, 10.0), name="random_feasible"):
    """Random sparse conic program, feasible and bounded by construction."""
    rng = np.random.default_rng(seed)
    soc_x, rsoc_x, socG, rsocG = list(soc_x), list(rsoc_x), list(socG), list(rsocG)
    n = n_box + sum(soc_x) + sum(rsoc_x) + 3 * (exp_x + dual_exp_x)
    m = mGzero + mGnonnegative + sum(socG) + sum(rsocG) + 3 * (expG + dual_expG)
    lo, hi = box
    # primal interior point
    parts = [rng.uniform(lo + 0.1 * (hi - lo), hi - 0.1 * (hi - lo), n_box)]
    parts += [_soc_interior(rng, d) for d in soc_x]
    parts += [_rsoc_interior(rng, d) for d in rsoc_x]
    parts += [_exp_interior(rng) for _ in range(exp_x)]
    parts += [_dexp_interior(rng) for _ in range(dual_exp_x)]
    x0 = np.concatenate(parts) if parts else np.zeros(0)
    # slack in int K_d and dual in int K_d^*
    s_parts = [np.zeros(mGzero), rng.uniform(0.1, 1.0, mGnonnegative)]
    y_parts = [rng.standard_normal(mGzero), rng.uniform(0.1, 1.0, mGnonnegative)]
    for d in socG:
        s_parts.append(_soc_interior(rng, d)); y_parts.append(_soc_interior(rng, d))
    for d in rsocG:
        s_parts.append(_rsoc_interior(rng, d)); y_parts.append(_rsoc_interior(rng, d))
    for _ in range(expG):
        s_parts.append(_exp_interior(rng)); y_parts.append(_dexp_interior(rng))
    for _ in range(dual_expG):
        s_parts.append(_dexp_interior(rng)); y_parts.append(_exp_interior(rng))
    s0 = np.concatenate(s_parts)
    y0 = np.concatenate(y_parts)
    # dual slack: free on a two-sided box, K_p^* interior on the cones
    l_parts = [rng.standard_normal(n_box)]
    l_parts += [_soc_interior(rng, d) for d in soc_x]
    l_parts += [_rsoc_interior(rng, d) for d in rsoc_x]
    l_parts += [_dexp_interior(rng) for _ in range(exp_x)]
    l_parts += [_exp_interior(rng) for _ in range(dual_exp_x)]
    lam0 = np.concatenate(l_parts) if l_parts else np.zeros(0)
    G = sp.random(m, n, density=density, format="csr", random_state=rng,
                  data_rvs=rng.standard_normal)
    G.sort_indices()
    h = G @ x0 - s0
    c = G.T @ y0 + lam0
    return ConicProblem(n=n, m=m, nb=n_box, c=c, G=G, h=h, mGzero=mGzero,
                        mGnonnegative=mGnonnegative, socG=socG, rsocG=rsocG, expG=expG,
                        dual_expG=dual_expG, bl=np.full(n_box, lo), bu=np.full(n_box, hi),
                        soc_x=soc_x, rsoc_x=rsoc_x, exp_x=exp_x, dual_exp_x=dual_exp_x,
                        name=name, seed=seed)


def socp_c0(seed=20261203, n_box=500, n_soc=500, m=800, density=0.01):
    """Random sparse SOCP: n = 1000 (500 boxed in [-10, 10], 500 in SOC blocks of
    dims uniform 3..10), m = 800 rows at 1% density with N(0, 1) values.
    K_d = 10% zero rows, 40% nonnegative rows, 50% in SOC blocks of dims 3..10."""
    rng = np.random.default_rng(seed + 7)
    soc_x = _random_dims(rng, n_soc, 3, 10)
    mz = m // 10
    mn = (4 * m) // 10
    socG = _random_dims(rng, m - mz - mn, 3, 10)
    return random_feasible(n_box=n_box, soc_x=soc_x, mGzero=mz, mGnonnegative=mn,
                           socG=socG, density=density, seed=seed, name="socp_c0")


def logreg_exp_c1(seed=20261204, samples=20000, features=500, density=0.05, lam=0.01):
    """l1-regularised logistic regression in exponential-cone form.

    min sum_i t_i + lam * sum_j (w+_j + w-_j)
    s.t. u_i + v_i <= 1,
         (-y_i a_i'(w+ - w-) - t_i, 1, u_i) in K_exp,   (-t_i, 1, v_i) in K_exp,
         w+, w- >= 0.
    x = [w+ (p) | w- (p) | t (N) | u (N) | v (N)], all in the box block;
    y = [N nonnegative rows | 2N exponential cones].
    Data: a_i with `density` nonzeros N(0, 1), labels +-1 Bernoulli(0.5)."""
    rng = np.random.default_rng(seed)
    N, p = samples, features
    A = sp.random(N, p, density=density, format="csr", random_state=rng,
                  data_rvs=rng.standard_normal)
    A.sort_indices()
    ylab = np.where(rng.random(N) < 0.5, -1.0, 1.0)
    n = 2 * p + 3 * N
    iw_p, iw_m, it, iu, iv = 0, p, 2 * p, 2 * p + N, 2 * p + 2 * N
    m = N + 6 * N
    rows, cols, vals = [], [], []
    h = np.zeros(m)
    ar = np.arange(N)
    # u_i + v_i <= 1  ->  -u_i - v_i + 1 >= 0
    rows += [ar, ar]; cols += [iu + ar, iv + ar]; vals += [-np.ones(N), -np.ones(N)]
    h[:N] = -1.0
    YA = sp.diags(ylab) @ A
    YA = YA.tocoo()
    base_a = N + 6 * ar            # first exp cone of sample i
    base_b = N + 6 * ar + 3        # second exp cone
    # cone a: (-y a'(w+ - w-) - t, 1, u)
    rows += [base_a[YA.row], base_a[YA.row], base_a]
    cols += [iw_p + YA.col, iw_m + YA.col, it + ar]
    vals += [-YA.data, YA.data, -np.ones(N)]
    h[base_a + 1] = -1.0
    rows += [base_a + 2]; cols += [iu + ar]; vals += [np.ones(N)]
    # cone b: (-t, 1, v)
    rows += [base_b]; cols += [it + ar]; vals += [-np.ones(N)]
    h[base_b + 1] = -1.0
    rows += [base_b + 2]; cols += [iv + ar]; vals += [np.ones(N)]
    G = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(m, n))
    G.sum_duplicates()
    G.sort_indices()
    c = np.concatenate([np.full(2 * p, lam), np.ones(N), np.zeros(2 * N)])
    bl = np.concatenate([np.zeros(2 * p), np.full(3 * N, -np.inf)])
    bu = np.full(n, np.inf)
    return ConicProblem(n=n, m=m, nb=n, c=c, G=G, h=h, mGzero=0, mGnonnegative=N,
                        expG=2 * N, bl=bl, bu=bu, name="logreg_exp_c1", seed=seed)


def mixed_small(seed=7, scale=1):
    """Small instance that exercises every cone type in K_d and K_p."""
    rng = np.random.default_rng(seed + 11)
    return random_feasible(
        n_box=20 * scale, soc_x=list(rng.integers(3, 7, 3 * scale)),
        rsoc_x=list(rng.integers(3, 6, 2 * scale)), exp_x=2 * scale, dual_exp_x=2 * scale,
        mGzero=5 * scale, mGnonnegative=15 * scale, socG=list(rng.integers(3, 7, 3 * scale)),
        rsocG=list(rng.integers(3, 6, 2 * scale)), expG=3 * scale, dual_expG=2 * scale,
        density=0.15, seed=seed, name="mixed_small")


def batch_socp_c3(count=4096, seed=20261206, nmin=50, nmax=5000, density=0.02):
    """Independent uneven SOCP instances, each built like socp_c0 with
    n log-uniform in [nmin, nmax], m = 0.8 n, SOC block dims uniform 3..20."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        n_box = n // 2
        m = max(int(0.8 * n), 10)
        r2 = np.random.default_rng(seed + 1000 + k)
        soc_x = _random_dims(r2, n - n_box, 3, 20)
        mz = m // 10
        mn = (4 * m) // 10
        socG = _random_dims(r2, m - mz - mn, 3, 20)
        out.append(random_feasible(n_box=n_box, soc_x=soc_x, mGzero=mz, mGnonnegative=mn,
                                   socG=socG, density=density, seed=seed + 1000 + k,
                                   name=f"batch_socp_{k}"))
    return out


def batch_mixed_c4(count=256, seed=20261207, n=2000, m=1500, density=0.01):
    """Mixed SOC + exponential-cone instances of equal size (the differentiable
    layer's workload): x = [box 800 | SOC blocks | 200 exp cones], y = [nonneg 300 |
    SOC blocks | 200 exp cones], each built feasible and bounded like socp_c0."""
    out = []
    for k in range(count):
        r2 = np.random.default_rng(seed + 7919 * k)
        n_exp, m_exp = n // 10, (2 * m) // 15
        n_box = (2 * n) // 5
        soc_x = _random_dims(r2, n - n_box - 3 * n_exp, 3, 10)
        mn = m // 5
        socG = _random_dims(r2, m - mn - 3 * m_exp, 3, 10)
        out.append(random_feasible(n_box=n_box, soc_x=soc_x, exp_x=n_exp, mGnonnegative=mn, socG=socG, expG=m_exp,
                                   density=density, seed=seed + 7919 * k, name=f"mixed_c4_{k}"))
    return out


def primal_infeasible_lp():
    """x1 + x2 >= 1 and -x1 - x2 >= 0 with x free: no feasible point."""
    G = sp.csr_matrix(np.array([[1.0, 1.0], [-1.0, -1.0], [1.0, 0.0]]))
    return ConicProblem(n=2, m=3, nb=2, c=np.array([1.0, 1.0]), G=G, h=np.array([1.0, 0.0, -5.0]),
                        mGzero=0, mGnonnegative=3, bl=np.full(2, -np.inf), bu=np.full(2, np.inf),
                        name="primal_infeasible_lp")


def dual_infeasible_lp():
    """min -x1 s.t. x1 - x2 >= 0, x2 >= 0, x free: unbounded below."""
    G = sp.csr_matrix(np.array([[1.0, -1.0], [0.0, 1.0]]))
    return ConicProblem(n=2, m=2, nb=2, c=np.array([-1.0, 0.0]), G=G, h=np.zeros(2),
                        mGzero=0, mGnonnegative=2, bl=np.full(2, -np.inf), bu=np.full(2, np.inf),
                        name="dual_infeasible_lp")


def portfolio_c2(n=1_000_000, factors=200, group=10, load_density=0.25, seed=20261205, gamma=1.0):
    """Robust portfolio with quadratic risk through a rotated second-order cone.

    Variables: the weights x (n, in [0, 1]) and the risk t >= 0 (nb = n + 1, all boxed).
        min  -mu'x + gamma t
        s.t. sum(x) = 1                                   (zero cone, 1 row)
             || x_g - w_g || <= r_g  for every group g    (n / group SOC blocks of dim group + 1)
             2 t (1/2) >= ||F'x||^2 + ||D x||^2          (one RSOC block of dim 2 + factors + n)
    F: factor loadings, each asset loading on a factor with probability
    load_density, values N(0, 0.1^2) (n = 1e6, 200 factors: about 5e7 nonzeros);
    D: idiosyncratic volatilities U(0.01, 0.1); mu ~ N(0.05, 0.02^2); w = 1/n
    (the benchmark, equal weights), r_g = 10 / n.  The equal-weight portfolio
    with t above its risk is an interior point, x is boxed and t >= 0 with
    gamma > 0, so the program is feasible and bounded."""
    rng = np.random.default_rng(seed)
    ng = n // group
    assert ng * group == n, "n must be a multiple of group"
    mu = rng.normal(0.05, 0.02, n)
    dvol = rng.uniform(0.01, 0.1, n)
    # rows of G in the layout [zero | SOC blocks | RSOC block]
    blocks = []
    # budget row
    blocks.append(sp.csr_matrix((np.ones(n), (np.zeros(n, dtype=np.int64), np.arange(n))), shape=(1, n + 1)))
    # tracking-error blocks: [r_g ; x_g - w_g] -> rows (empty, then the identity on x_g)
    rows = np.arange(ng * (group + 1)).reshape(ng, group + 1)[:, 1:].ravel()
    blocks.append(sp.csr_matrix((np.ones(n), (rows, np.arange(n))), shape=(ng * (group + 1), n + 1)))
    # risk block: [t ; 1/2 ; F'x ; D x]
    fr, fc, fv = [], [], []
    for f in range(factors):
        cols = np.nonzero(rng.random(n) < load_density)[0]
        fr.append(np.full(cols.size, 2 + f, dtype=np.int64))
        fc.append(cols)
        fv.append(rng.normal(0.0, 0.1, cols.size))
    r_rows = np.concatenate([[0]] + fr + [2 + factors + np.arange(n)])
    r_cols = np.concatenate([[n]] + fc + [np.arange(n)])
    r_vals = np.concatenate([[1.0]] + fv + [dvol])
    blocks.append(sp.csr_matrix((r_vals, (r_rows, r_cols)), shape=(2 + factors + n, n + 1)))
    G = sp.vstack(blocks, format="csr")
    G.sort_indices()
    m = G.shape[0]
    h = np.zeros(m)
    h[0] = 1.0
    r_g = 10.0 / n
    soc_rows = 1 + np.arange(ng) * (group + 1)
    h[soc_rows] = -r_g
    h[(soc_rows[:, None] + 1 + np.arange(group)[None, :]).ravel()] = 1.0 / n
    rs = 1 + ng * (group + 1)
    h[rs + 1] = -0.5
    c = np.concatenate([-mu, [gamma]])
    bl = np.zeros(n + 1)
    bu = np.concatenate([np.ones(n), [np.inf]])
    return ConicProblem(n=n + 1, m=m, nb=n + 1, c=c, G=G, h=h, mGzero=1, mGnonnegative=0,
                        socG=[group + 1] * ng, rsocG=[2 + factors + n], bl=bl, bu=bu,
                        name=f"portfolio_c2_{n}", seed=seed)
