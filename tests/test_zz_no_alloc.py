"""pdcs_spmv_csr_noalloc: the SpMV entry point for callers that cannot allocate.

Callers whose device memory is owned by their own pool allocator, or that run
latency-critical loops, cannot have the library call cudaMalloc; this entry
point keeps its row-carry scratch in a fixed device array instead.  The test
calls it through the C ABI twice in a row (different matrices, so the second
call runs on the scratch the first one left behind) and checks each result
against pdcs_spmv_csr.  It lives in its own file, collected last, and passes
both alone in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

LIMIT_STATUS = -10  # PDCS_ERR_NOALLOC_LIMIT


def _device_csr(A, x, dev):
    import torch
    t = lambda a, dt: torch.as_tensor(a, dtype=dt, device=dev)
    return (t(A.indptr, torch.int32), t(A.indices, torch.int32), t(A.data, torch.float64),
            t(x, torch.float64))


def _call(fn, A, bufs, y):
    rp, ci, v, xt = bufs
    return fn(A.shape[0], A.shape[1], A.nnz, rp.data_ptr(), ci.data_ptr(), v.data_ptr(), xt.data_ptr(),
              y.data_ptr(), None)


def test_noalloc_matches_allocating_entry_point_twice(cuda):
    import torch
    from pdcs_b200 import capi
    lib = capi.load()
    rng = np.random.default_rng(2026)
    mats = [sp.random(5000, 3000, density=0.01, format="csr", random_state=rng, data_rvs=rng.standard_normal),
            sp.random(700, 90000, density=0.05, format="csr", random_state=rng, data_rvs=rng.standard_normal)]
    for A in mats:
        A.sort_indices()
        x = rng.standard_normal(A.shape[1])
        bufs = _device_csr(A, x, cuda)
        y_ref = torch.full((A.shape[0],), float("nan"), dtype=torch.float64, device=cuda)
        y_new = torch.full((A.shape[0],), float("nan"), dtype=torch.float64, device=cuda)
        assert _call(lib.pdcs_spmv_csr, A, bufs, y_ref) == 0
        assert _call(lib.pdcs_spmv_csr_noalloc, A, bufs, y_new) == 0
        torch.cuda.synchronize()
        a, b = y_new.cpu().numpy(), y_ref.cpu().numpy()
        assert np.all(np.isfinite(a))
        assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(b).max()))
        assert np.allclose(a, A @ x, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(b).max()))


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    from pdcs_b200 import capi
    lib = capi.load()
    buf = torch.zeros(8, dtype=torch.float64, device=cuda)
    ibuf = torch.zeros(8, dtype=torch.int32, device=cuda)
    m = 134217728  # m + nnz just above the 65536 x 2048 merge items of the fixed scratch
    rc = lib.pdcs_spmv_csr_noalloc(m, 1, 1, ibuf.data_ptr(), ibuf.data_ptr(), buf.data_ptr(), buf.data_ptr(),
                                   buf.data_ptr(), None)
    assert rc == LIMIT_STATUS


def test_noalloc_empty_rows_at_cta_boundaries_and_no_nonzeros(cuda):
    """Rows without nonzeros where the merge path splits CTAs (2048 merge
    items, one per row end and one per nonzero, per CTA), a row that spans
    several CTAs, and a matrix with no nonzeros at all (NULL column indices,
    values and x).  Each result is compared with pdcs_spmv_csr and A @ x."""
    import torch
    from pdcs_b200 import capi
    lib = capi.load()
    rng = np.random.default_rng(7)
    lens = [0] * 2040 + [5] + [0] * 10 + [4000] + [0] * 3000 + [1] * 100 + [0] * 2100 + [3] + [0] * 2047
    n = 6000
    indptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    indices = np.concatenate([np.sort(rng.choice(n, k, replace=False)) for k in lens if k]).astype(np.int32)
    A = sp.csr_matrix((rng.standard_normal(indptr[-1]), indices, indptr), shape=(len(lens), n))
    x = rng.standard_normal(n)
    bufs = _device_csr(A, x, cuda)
    for _ in range(2):
        y_ref = torch.full((A.shape[0],), float("nan"), dtype=torch.float64, device=cuda)
        y_new = torch.full((A.shape[0],), float("nan"), dtype=torch.float64, device=cuda)
        assert _call(lib.pdcs_spmv_csr, A, bufs, y_ref) == 0
        assert _call(lib.pdcs_spmv_csr_noalloc, A, bufs, y_new) == 0
        torch.cuda.synchronize()
        a, b = y_new.cpu().numpy(), y_ref.cpu().numpy()
        assert np.all(np.isfinite(a))
        assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(b).max()))
        assert np.allclose(a, A @ x, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(b).max()))
    m = 5000
    rp = torch.zeros(m + 1, dtype=torch.int32, device=cuda)
    for _ in range(2):
        y = torch.full((m,), float("nan"), dtype=torch.float64, device=cuda)
        assert lib.pdcs_spmv_csr_noalloc(m, 7, 0, rp.data_ptr(), None, None, None, y.data_ptr(), None) == 0
        torch.cuda.synchronize()
        assert torch.count_nonzero(y).item() == 0
