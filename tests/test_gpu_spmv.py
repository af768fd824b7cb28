"""pdcs_spmv_csr vs scipy on matrices with empty, short and long rows."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,density", [((1000, 700), 0.01), ((300, 5000), 0.3), ((5, 20000), 0.5),
                                           ((20000, 50), 0.02)])
def test_spmv_matches_scipy(cuda, shape, density):
    import torch
    from pdcs_b200 import capi
    rng = np.random.default_rng(shape[0])
    A = sp.random(*shape, density=density, format="csr", random_state=rng, data_rvs=rng.standard_normal)
    A.sort_indices()
    x = rng.standard_normal(shape[1])
    t = lambda a, dt: torch.as_tensor(a, dtype=dt, device=cuda)
    rp, ci, v, xt = t(A.indptr, torch.int32), t(A.indices, torch.int32), t(A.data, torch.float64), t(x, torch.float64)
    y = torch.empty(shape[0], dtype=torch.float64, device=cuda)
    rc = capi.load().pdcs_spmv_csr(shape[0], shape[1], A.nnz, rp.data_ptr(), ci.data_ptr(), v.data_ptr(),
                                   xt.data_ptr(), y.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    ref = A @ x
    assert np.allclose(y.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def _skewed(rng):
    """Empty leading/trailing rows, one 300k-nnz row spanning many CTAs, short rows."""
    import scipy.sparse as sp
    m, n = 4000, 400000
    rows, cols = [], []
    long_cols = rng.choice(n, 300000, replace=False)
    rows.append(np.full(long_cols.size, 1700)); cols.append(long_cols)
    for r in range(10, 3990, 3):
        k = int(rng.integers(0, 6))
        rows.append(np.full(k, r)); cols.append(rng.choice(n, k, replace=False))
    r = np.concatenate(rows); c = np.concatenate(cols)
    A = sp.csr_matrix((rng.standard_normal(r.size), (r, c)), shape=(m, n))
    A.sum_duplicates(); A.sort_indices()
    return A


def test_spmv_skewed_rows(cuda):
    import torch
    from pdcs_b200 import capi
    rng = np.random.default_rng(7)
    A = _skewed(rng)
    x = rng.standard_normal(A.shape[1])
    t = lambda a, dt: torch.as_tensor(a, dtype=dt, device=cuda)
    rp, ci, v, xt = t(A.indptr, torch.int32), t(A.indices, torch.int32), t(A.data, torch.float64), t(x, torch.float64)
    y = torch.full((A.shape[0],), float("nan"), dtype=torch.float64, device=cuda)
    rc = capi.load().pdcs_spmv_csr(A.shape[0], A.shape[1], A.nnz, rp.data_ptr(), ci.data_ptr(), v.data_ptr(),
                                   xt.data_ptr(), y.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    ref = A @ x
    assert np.allclose(y.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
