"""Solution-map adjoint (pdcs_grad / pdcs_batch_grad) and the torch layer.

The GPU adjoint (restarted GMRES on (I - M)' u = g with the projection-Jacobian
kernels) is checked against (1) the dense FP64 reference of the same
fixed-point derivative (tests/_adjoint_reference.py) at the same solution and
step sizes, (2) the dense FP64 derivative of the conic KKT conditions, which
involves no step sizes, (3) central finite differences of GPU solves (step
1e-6, FP64), also on one instance of the differentiable layer's size
(n = 2000, m = 1500), and (4) batched vs single calls."""
import copy

import numpy as np
import pytest
import scipy.sparse as sp

import _adjoint_reference as R
from pdcs_b200 import problems, solver

pytestmark = pytest.mark.gpu

# 1e-9: below ~1e-10 a restart at an almost exact solution lets the adaptive step grow
# on rounding noise and the iteration can diverge (the reference's algorithm does too)
TIGHT = dict(rel_tol=1e-9, abs_tol=1e-9, time_limit=120)


def _instances():
    tight_box = problems.mixed_small(seed=5)
    tight_box.c = tight_box.c.copy()
    tight_box.c[:tight_box.nb] += 4.0 * np.sign(np.random.default_rng(1).standard_normal(tight_box.nb))
    tight_box.name = "mixed_active_box"
    return [problems.mixed_small(),
            problems.random_feasible(n_box=8, soc_x=[3, 4], rsoc_x=[3], exp_x=1, dual_exp_x=1, mGzero=2,
                                     mGnonnegative=5, socG=[3, 4], rsocG=[3], expG=1, dual_expG=1, density=0.5,
                                     seed=3, name="tiny_mixed"),
            problems.socp_c0(n_box=40, n_soc=40, m=60, density=0.1, seed=4),
            tight_box]


@pytest.mark.parametrize("idx", range(4))
def test_grad_matches_dense_reference(cuda, idx):
    p = _instances()[idx]
    s = solver.solve_problem(p, **TIGHT)
    assert s.info.exit_status == "optimal"
    xt = np.random.default_rng(idx).standard_normal(p.n)
    g, info = solver.rpdhg_gpu_grad(p, s.primal, s.dual, s.primal - xt)
    assert info.converged, info
    ref = R.adjoint_dense(p, s.primal, s.dual, s.primal - xt)  # the same steps as the GPU adjoint
    for key in ("c", "h", "G", "bl", "bu"):
        scale = max(1e-12, np.abs(ref[key]).max()) if ref[key].size else 1.0
        err = np.abs(g[key] - ref[key]).max() / scale if ref[key].size else 0.0
        print(p.name, key, f"max rel err vs dense FP64 reference {err:.2e}")
        assert err <= 1e-6, (p.name, key, err)


@pytest.mark.parametrize("idx", range(4))
def test_grad_matches_kkt_reference(cuda, idx):
    p = _instances()[idx]
    s = solver.solve_problem(p, **TIGHT)
    assert s.info.exit_status == "optimal"
    xt = np.random.default_rng(10 + idx).standard_normal(p.n)
    g, info = solver.rpdhg_gpu_grad(p, s.primal, s.dual, s.primal - xt)
    assert info.converged, info
    ref = R.adjoint_kkt(p, s.primal, s.dual, s.primal - xt)
    for key in ("c", "h", "G", "bl", "bu"):
        if not ref[key].size:
            continue
        err = np.abs(g[key] - ref[key]).max() / max(1e-12, np.abs(ref[key]).max())
        print(p.name, key, f"max rel err vs the KKT-derivative reference {err:.2e}")
        assert err <= 1e-6, (p.name, key, err)


def _c4_instance():
    return problems.batch_mixed_c4(count=1, seed=20261207)[0]


@pytest.mark.parametrize("which", ["small", "c4"])
def test_grad_matches_finite_differences(cuda, which):
    p = _instances()[0] if which == "small" else _c4_instance()
    s = solver.solve_problem(p, **TIGHT)
    rng = np.random.default_rng(7)
    xt = rng.standard_normal(p.n)
    g, _ = solver.rpdhg_gpu_grad(p, s.primal, s.dual, s.primal - xt)

    def loss(q):
        r = solver.solve_problem(q, **TIGHT)
        assert r.info.exit_status == "optimal"
        return 0.5 * np.sum((r.primal - xt) ** 2)
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
        err = abs(fd - an) / max(1e-12, abs(fd))
        print(f"{key}: central difference {fd:.8e} adjoint {an:.8e} rel err {err:.2e}")
        assert err <= 1e-4, (key, fd, an)


def test_batched_grad_matches_single(cuda):
    batch = _instances()
    with solver.BatchHandle(batch, differentiable=True, **TIGHT) as h:
        sols, _ = h.solve()
        rng = np.random.default_rng(3)
        gx = [rng.standard_normal(p.n) for p in batch]
        grads, infos = h.grad(gx)
    for p, s, gi, g, inf in zip(batch, sols, gx, grads, infos):
        assert inf.converged, (p.name, inf)
        one, _ = solver.rpdhg_gpu_grad(p, s.primal, s.dual, gi)
        for key in g:
            scale = max(1e-12, np.abs(one[key]).max()) if one[key].size else 1.0
            assert np.abs(g[key] - one[key]).max() <= 1e-7 * scale, (p.name, key)


def test_torch_layer_backward(cuda):
    import torch
    from pdcs_b200.autograd import ConicBatchLayer
    batch = _instances()[:3]
    layer = ConicBatchLayer(batch, **TIGHT)
    c, h, gv, bl, bu = [t.requires_grad_() for t in layer.flat_params(batch)]
    xt = torch.randn(sum(p.n for p in batch), dtype=torch.float64, generator=torch.Generator().manual_seed(0))
    x = layer(c, h, gv, bl, bu)
    loss = 0.5 * ((x - xt) ** 2).sum()
    loss.backward()
    off = 0
    for p in batch:
        s = solver.solve_problem(p, **TIGHT)
        one, _ = solver.rpdhg_gpu_grad(p, s.primal, s.dual, s.primal - xt[off:off + p.n].numpy())
        got = c.grad[off:off + p.n].numpy()
        assert np.abs(got - one["c"]).max() <= 1e-5 * max(1.0, np.abs(one["c"]).max()), p.name
        off += p.n


def test_c4_size_grad_matches_kkt_reference(cuda):
    """One instance of the differentiable layer's workload (n = 2000, m = 1500,
    1% density, SOC + exponential cones): the GPU adjoint against the dense
    step-free KKT derivative."""
    p = _c4_instance()
    s = solver.solve_problem(p, **TIGHT)
    assert s.info.exit_status == "optimal"
    xt = np.random.default_rng(5).standard_normal(p.n)
    g, info = solver.rpdhg_gpu_grad(p, s.primal, s.dual, s.primal - xt)
    assert info.converged, info
    ref = R.adjoint_kkt(p, s.primal, s.dual, s.primal - xt)
    for key in ("c", "h", "G", "bl", "bu"):
        err = np.abs(g[key] - ref[key]).max() / max(1e-12, np.abs(ref[key]).max())
        print(p.name, key, f"max rel err vs the KKT-derivative reference {err:.2e}")
        assert err <= 1e-6, (key, err)
