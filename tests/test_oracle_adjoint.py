"""The dense FP64 references of the solution-map adjoint (tests/_adjoint_reference.py):
the PDHG fixed-point derivative with the GPU adjoint's step sizes
(adjoint_dense) against the step-free conic-KKT derivative (adjoint_kkt), and
both against central finite differences of the oracle solver (CPU)."""
import pytest
import copy

import numpy as np
import scipy.sparse as sp

import _adjoint_reference as R
from pdcs_b200 import problems


def test_dense_adjoint_matches_oracle_finite_differences():
    p = problems.mixed_small()
    x, y, r = R.solve_tight(p)
    assert r["exit_code"] == 0
    rng = np.random.default_rng(1)
    xt = rng.standard_normal(p.n)
    g = R.adjoint_dense(p, x, y, x - xt)

    def loss(q):
        xx, _, rr = R.solve_tight(q)
        assert rr["exit_code"] == 0
        return 0.5 * np.sum((xx - xt) ** 2)
    eps = 1e-6
    for key in ("c", "h", "G"):
        d = rng.standard_normal(len(g[key]))
        q1, q2 = copy.deepcopy(p), copy.deepcopy(p)
        if key == "G":
            G = sp.csr_matrix(p.G)
            G.sort_indices()
            q1.G = sp.csr_matrix((G.data + eps * d, G.indices, G.indptr), shape=G.shape)
            q2.G = sp.csr_matrix((G.data - eps * d, G.indices, G.indptr), shape=G.shape)
        else:
            setattr(q1, key, getattr(p, key) + eps * d)
            setattr(q2, key, getattr(p, key) - eps * d)
        fd = (loss(q1) - loss(q2)) / (2 * eps)
        an = float(g[key] @ d)
        assert abs(fd - an) <= 1e-4 * max(1e-12, abs(fd)), (key, fd, an)
        an_kkt = float(R.adjoint_kkt(p, x, y, x - xt)[key] @ d)
        assert abs(fd - an_kkt) <= 1e-4 * max(1e-12, abs(fd)), (key, fd, an_kkt)


def test_projection_jacobians_match_differences():
    """Closed-form cone Jacobians against central differences of the oracle's projections."""
    rng = np.random.default_rng(2)
    for kind, d, jac in (("soc", 5, R.soc_jac), ("rsoc", 5, R.rsoc_jac), ("exp", 3, R.exp_jac)):
        for _ in range(20):
            a = rng.standard_normal(d) * 2.0
            J = jac(a)
            eps = 1e-7
            Jfd = np.zeros((d, d))
            for i in range(d):
                e = np.zeros(d)
                e[i] = eps
                from oracle import binding as B
                Jfd[:, i] = (B.project_block(kind, a + e) - B.project_block(kind, a - e)) / (2 * eps)
            assert np.abs(J - Jfd).max() <= 1e-5 * max(1.0, np.abs(J).max()), (kind, a)


def _instances():
    return [problems.mixed_small(),
            problems.random_feasible(n_box=8, soc_x=[3, 4], rsoc_x=[3], exp_x=1, dual_exp_x=1, mGzero=2,
                                     mGnonnegative=5, socG=[3, 4], rsocG=[3], expG=1, dual_expG=1, density=0.5,
                                     seed=3, name="tiny_mixed"),
            problems.socp_c0(n_box=40, n_soc=40, m=60, density=0.1, seed=4)]


@pytest.mark.parametrize("idx", range(3))
def test_fixed_point_derivative_equals_kkt_derivative(idx):
    """The fixed-point derivative with Pock-Chambolle steps and the step-free
    KKT derivative are the same map: they agree to rounding."""
    p = _instances()[idx]
    x, y, r = R.solve_tight(p)
    assert r["exit_code"] == 0
    xt = np.random.default_rng(idx).standard_normal(p.n)
    a = R.adjoint_dense(p, x, y, x - xt)
    b = R.adjoint_kkt(p, x, y, x - xt)
    for key in a:
        if a[key].size:
            scale = max(1e-12, np.abs(b[key]).max())
            assert np.abs(a[key] - b[key]).max() <= 1e-8 * scale, (p.name, key)
