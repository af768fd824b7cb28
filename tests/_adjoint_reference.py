"""Dense FP64 reference of the solution-map adjoint (test infrastructure).

The solution (x*, y*) of min c'x s.t. Gx - h in K_d, x in X = box x K_p is a
fixed point of the PDHG map T for positive diagonal steps T, S constant on
every cone block:
    x+ = P_X(x + T (G'y - c)),   y+ = P_{K_d*}(y - S (G (2 x+ - x) - h)).
With M = dT/dz at the fixed point, dz*/dtheta = (I - M)^{-1} dT/dtheta, so for
a loss L(x*, y*) with g = dL/dz*, u solves (I - M)' u = g and
    w = D_K u_y,  q = u_x - 2 G' (S w),  r = D_X q,
    dL/dc = -T r,  dL/dh = S w,  dL/dG_ij = T_j y_i r_j - S_i w_i x_j,
    dL/dl_j = q_j [a_j < l_j],  dL/du_j = q_j [a_j > u_j]
(D_X, D_K: Jacobians of the projections at a = x + T (G'y - c) and
b = y - S (G x - h)).  The default steps are the GPU adjoint's: 0.9 / column
(row) absolute sums of G, at their minimum over each cone block.  Here every piece is a dense numpy matrix; the
projections come from the oracle and their Jacobians from closed forms
written independently of the CUDA kernels.
"""
import numpy as np
import scipy.sparse as sp

from oracle import binding as B


def blocks(p, side):
    """(kind, start, length) of the cones of x (side "x": X = box x K_p) or of
    the dual cone K_d* of y (side "y")."""
    out = []
    if side == "x":
        if p.nb:
            out.append(("BOX", 0, p.nb))
        s = p.nb
        for d in p.soc_x:
            out.append(("SOC", s, d)); s += d
        for d in p.rsoc_x:
            out.append(("RSOC", s, d)); s += d
        for _ in range(p.exp_x):
            out.append(("EXP", s, 3)); s += 3
        for _ in range(p.dual_exp_x):
            out.append(("DEXP", s, 3)); s += 3
        if s < p.n:
            out.append(("FREE", s, p.n - s))
    else:
        s = 0
        if p.mGzero:
            out.append(("FREE", 0, p.mGzero)); s = p.mGzero
        if p.mGnonnegative:
            out.append(("NONNEG", s, p.mGnonnegative)); s += p.mGnonnegative
        for d in p.socG:
            out.append(("SOC", s, d)); s += d
        for d in p.rsocG:
            out.append(("RSOC", s, d)); s += d
        for _ in range(p.expG):
            out.append(("DEXP", s, 3)); s += 3  # dual of the exponential cone
        for _ in range(p.dual_expG):
            out.append(("EXP", s, 3)); s += 3
    return out


def project(p, side, v):
    out = np.array(v, dtype=np.float64)
    for kind, s, d in blocks(p, side):
        if kind == "BOX":
            out[s:s + d] = np.clip(v[s:s + d], p.bl, p.bu)
        elif kind == "FREE":
            pass
        elif kind == "NONNEG":
            out[s:s + d] = np.maximum(v[s:s + d], 0.0)
        else:
            out[s:s + d] = B.project_block(kind.lower(), v[s:s + d])
    return out


def soc_jac(a):
    t, x = a[0], a[1:]
    nx = np.linalg.norm(x)
    d = len(a)
    if nx <= t:
        return np.eye(d)
    if nx <= -t:
        return np.zeros((d, d))
    xh = x / nx
    J = np.zeros((d, d))
    J[0, 0] = 1.0
    J[0, 1:] = xh
    J[1:, 0] = xh
    J[1:, 1:] = (1.0 + t / nx) * np.eye(d - 1) - (t / nx) * np.outer(xh, xh)
    return 0.5 * J


def rsoc_jac(a):
    d = len(a)
    R = np.eye(d)
    R[:2, :2] = np.array([[1.0, 1.0], [1.0, -1.0]]) / np.sqrt(2.0)
    return R @ soc_jac(R @ a) @ R


def exp_jac(a):
    p = B.project_block("exp", a)
    r, s, t = p
    scale = 1.0 + np.linalg.norm(a)
    if np.linalg.norm(p - a) <= 1e-13 * scale:
        return np.eye(3)
    if np.linalg.norm(p) <= 1e-13 * scale:
        return np.zeros((3, 3))
    if s <= 1e-13 * scale:  # r <= 0, s <= 0 region: p = (r, 0, max(t, 0))
        return np.diag([1.0, 0.0, 1.0 if a[2] > 0 else 0.0])
    rho = r / s
    e = np.exp(rho)
    g = np.array([e, e * (1.0 - rho), -1.0])
    Hs = (e / s) * np.array([[1.0, -rho, 0.0], [-rho, rho * rho, 0.0], [0.0, 0.0, 0.0]])
    mu = float((a - p) @ g) / float(g @ g)
    Bm = np.eye(3) + mu * Hs
    Bi = np.linalg.inv(Bm)
    bg = Bi @ g
    return Bi - np.outer(bg, bg) / float(g @ bg)


def jacobian(p, side, a):
    n = len(a)
    J = np.zeros((n, n))
    for kind, s, d in blocks(p, side):
        v = a[s:s + d]
        if kind == "BOX":
            J[s:s + d, s:s + d] = np.diag(((v > p.bl) & (v < p.bu)).astype(float))
        elif kind == "FREE":
            J[s:s + d, s:s + d] = np.eye(d)
        elif kind == "NONNEG":
            J[s:s + d, s:s + d] = np.diag((v > 0).astype(float))
        elif kind == "SOC":
            J[s:s + d, s:s + d] = soc_jac(v)
        elif kind == "RSOC":
            J[s:s + d, s:s + d] = rsoc_jac(v)
        elif kind == "EXP":
            J[s:s + d, s:s + d] = exp_jac(v)
        elif kind == "DEXP":  # Moreau: P_{K*}(v) = v + P_K(-v)
            J[s:s + d, s:s + d] = np.eye(3) - exp_jac(-v)
    return J


def default_steps(p):
    """T (n) and S (m): 0.9 / absolute column (row) sums of G (1 where 0), at
    their minimum over every cone block that is not elementwise."""
    A = abs(sp.csr_matrix(p.G))
    cs = np.asarray(A.sum(axis=0)).ravel()
    rs = np.asarray(A.sum(axis=1)).ravel()
    T = np.where(cs > 0, 0.9 / np.where(cs > 0, cs, 1.0), 1.0)
    S = np.where(rs > 0, 0.9 / np.where(rs > 0, rs, 1.0), 1.0)
    for side, d in (("x", T), ("y", S)):
        for kind, s, L in blocks(p, side):
            if kind in ("SOC", "RSOC", "EXP", "DEXP"):
                d[s:s + L] = d[s:s + L].min()
    return T, S


def adjoint_dense(p, x, y, gx, gy=None, T=None, S=None):
    """Gradients of L at the solution (x, y) given g = (dL/dx*, dL/dy*): dict of c, h, G (nzval
    in the CSR order of p.G), bl, bu."""
    G = sp.csr_matrix(p.G)
    G.sort_indices()
    Gd = G.toarray()
    if T is None:
        T, S = default_steps(p)
    a = x + T * (Gd.T @ y - p.c)
    xp = project(p, "x", a)
    b = y - S * (Gd @ (2 * xp - x) - p.h)
    DX = jacobian(p, "x", a)
    DK = jacobian(p, "y", b)
    n, m = p.n, p.m
    SG = S[:, None] * Gd
    TGt = T[:, None] * Gd.T
    M = np.zeros((n + m, n + m))
    M[:n, :n] = DX
    M[:n, n:] = DX @ TGt
    M[n:, :n] = DK @ SG @ (np.eye(n) - 2 * DX)
    M[n:, n:] = DK @ (np.eye(m) - 2 * SG @ DX @ TGt)
    g = np.concatenate([gx, np.zeros(m) if gy is None else gy])
    u = np.linalg.lstsq((np.eye(n + m) - M).T, g, rcond=None)[0]
    ux, uy = u[:n], u[n:]
    w = DK @ uy
    t1 = Gd.T @ (S * w)
    q = ux - 2 * t1
    r = DX @ q
    rows = np.repeat(np.arange(m), np.diff(G.indptr))
    cols = G.indices
    dG = T[cols] * y[rows] * r[cols] - S[rows] * w[rows] * x[cols]
    lo = a[:p.nb] < p.bl
    hi = a[:p.nb] > p.bu
    return {"c": -T * r, "h": S * w, "G": dG, "bl": q[:p.nb] * lo, "bu": q[:p.nb] * hi}


def solve_tight(p, **kw):
    """The oracle's solution to 1e-9 (in practice ~1e-11: the criteria are checked
    every 2000 attempts; tighter requests can end in the adaptive step's divergence)."""
    r = B.solve(p, threads=1, rel_tol=1e-9, abs_tol=1e-9, **kw)
    return r["x"], r["y"], r


def adjoint_kkt(p, x, y, gx, gy=None):
    """Gradients of L from the conic KKT conditions, independent of any step
    sizes: (x, y) is optimal iff F(z) = 0 with
        F_x = x - P_X(a),      a = x - (c - G'y)   (-(c - G'y) in N_X(x)),
        F_y = y - P_{K_d*}(b), b = y - (G x - h)   (Gx - h in K_d, y in K_d*, <y, Gx - h> = 0),
    so dz*/dtheta = -(dF/dz)^{-1} dF/dtheta and, with v solving
    (dF/dz)' v = g,
        dL/dc = -D_X v_x,  dL/dh = D_K v_y,
        dL/dG_ij = (D_X v_x)_j y_i - (D_K v_y)_i x_j,
        dL/dl_j = v_x,j [a_j < l_j],  dL/du_j = v_x,j [a_j > u_j]
    (D_X, D_K: the projections' Jacobians at a and b, symmetric).  Dense
    FP64 throughout; nothing is shared with the PDHG fixed-point form but the
    projections and their Jacobians."""
    G = sp.csr_matrix(p.G)
    G.sort_indices()
    Gd = G.toarray()
    n, m = p.n, p.m
    a = x - (p.c - Gd.T @ y)
    b = y - (Gd @ x - p.h)
    DX = jacobian(p, "x", a)
    DK = jacobian(p, "y", b)
    J = np.zeros((n + m, n + m))
    J[:n, :n] = np.eye(n) - DX
    J[:n, n:] = -DX @ Gd.T
    J[n:, :n] = DK @ Gd
    J[n:, n:] = np.eye(m) - DK
    g = np.concatenate([gx, np.zeros(m) if gy is None else gy])
    v = np.linalg.lstsq(J.T, g, rcond=None)[0]
    vx, vy = v[:n], v[n:]
    ax = DX @ vx
    ky = DK @ vy
    rows = np.repeat(np.arange(m), np.diff(G.indptr))
    cols = G.indices
    lo = a[:p.nb] < p.bl
    hi = a[:p.nb] > p.bu
    return {"c": -ax, "h": ky, "G": ax[cols] * y[rows] - ky[rows] * x[cols],
            "bl": vx[:p.nb] * lo, "bu": vx[:p.nb] * hi}
