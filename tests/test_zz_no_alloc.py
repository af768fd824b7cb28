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
