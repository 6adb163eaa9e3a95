"""The allocation-free entry point against the allocating one (needs a B200).

Some callers of this library cannot allocate device memory. Code inside
another framework's custom-call or FFI handler may only use the buffers it is
handed. A host may reserve all device memory up front. Code may be unable to
call cudaMalloc while a CUDA graph is being captured. For them the library has
one entry point, ``pb_integrate_const_noalloc``, whose scratch is a fixed,
file-scope device array.

This test calls it through the C ABI with caller-owned device buffers. It
checks the result against ``pb_integrate_const`` on two calls in a row: the
second call starts from whatever the first left in the shared scratch. It also
checks that sizes beyond the static limit are rejected.
"""

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu
TOL = 1e-10
MAX_STATES = 65536


def _case(n, seed):
    """A decaying operator: negative diagonal, non-negative off-diagonal feed."""
    rng = np.random.default_rng(seed)
    d = -rng.uniform(0.05, 2.0, n)
    if n <= 3:
        L = sp.csr_matrix(np.diag(np.full(n - 1, 0.7), -1)) if n > 1 else sp.csr_matrix((n, n))
    else:
        rows = rng.integers(0, n, 6 * n)
        cols = rng.integers(0, n, 6 * n)
        keep = rows != cols
        L = sp.csr_matrix((rng.uniform(0.0, 0.2, keep.sum()), (rows[keep], cols[keep])), shape=(n, n))
        L.sum_duplicates()
        L.sort_indices()
    zg = np.linspace(0.0, 3.0, 301)
    x0 = rng.uniform(0.5, 1.5, n)
    return d, L, zg, x0


def _device(a, dtype):
    import torch

    return torch.tensor(np.ascontiguousarray(a, dtype=dtype), device="cuda:0")


@pytest.mark.parametrize("n,seed", [(3, 0), (5000, 1)])
def test_noalloc_matches_allocating_entry_point(n, seed):
    import torch
    from prince_b200 import _lib

    ctx = _lib.Context(0)
    d, L, zg, x0 = _case(n, seed)
    ref = ctx.integrate_const(d, L, zg, x0)
    td = _device(d, np.float64)
    tip = _device(L.indptr, np.int64)
    tix = _device(L.indices if L.nnz else np.zeros(1), np.int32)
    tv = _device(L.data if L.nnz else np.zeros(1), np.float64)
    tz = _device(zg, np.float64)
    for _ in range(2):
        tx = _device(x0, np.float64)
        torch.cuda.synchronize()
        ctx.integrate_const_noalloc(n, td.data_ptr(), L.nnz, tip.data_ptr(), tix.data_ptr(), tv.data_ptr(),
                                    zg.size - 1, tz.data_ptr(), tx.data_ptr())
        out = tx.cpu().numpy()
        np.testing.assert_allclose(out, ref, rtol=TOL, atol=0)


def test_noalloc_rejects_sizes_beyond_the_static_limit():
    from prince_b200 import _lib

    ctx = _lib.Context(0)
    buf = _device(np.zeros(4), np.float64)
    p = buf.data_ptr()
    with pytest.raises(ValueError, match="static scratch limit"):
        ctx.integrate_const_noalloc(MAX_STATES + 1, p, 0, None, None, None, 1, p, p)
    with pytest.raises(ValueError, match="static scratch limit"):
        ctx.integrate_const_noalloc(2, p, 0, None, None, None, 16385, p, p)
