"""The dense FP64 reference of the solution-map adjoint (tests/_adjoint_reference.py)
against central finite differences of the oracle solver (CPU; pins the
fixed-point derivative the GPU adjoint implements)."""
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
        assert abs(fd - an) <= 1e-3 * max(1e-12, abs(fd)), (key, fd, an)


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
