"""The allocation-free entry point against the allocating one (needs a B200).

Some callers of this library cannot allocate device memory. Code inside
another framework's custom-call or FFI handler may only use the buffers it is
handed, and a host may have reserved all device memory up front. For them the
library has one entry point, ``pb_integrate_const_noalloc``, whose scratch is a
fixed, file-scope device array.

This test calls it through the C ABI with caller-owned device buffers. It
checks the result against ``pb_integrate_const`` on two calls in a row (the
second call starts from whatever the first left in the shared scratch), for an
operator with no off-diagonal entries (row pointers passed as NULL), for zero
steps and at the state limit. It also checks that sizes beyond the static limit
and malformed CSR arrays are rejected before any step runs.
"""

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu
TOL = 1e-10
MAX_STATES = 65536
MAX_STEPS = 16384


def _case(n, seed, n_steps=300, offdiag=True):
    """A decaying operator: negative diagonal, non-negative off-diagonal feed."""
    rng = np.random.default_rng(seed)
    d = -rng.uniform(0.05, 2.0, n)
    if not offdiag:
        L = sp.csr_matrix((n, n))
    elif n <= 3:
        L = sp.csr_matrix(np.diag(np.full(n - 1, 0.7), -1)) if n > 1 else sp.csr_matrix((n, n))
    else:
        rows = rng.integers(0, n, 6 * n)
        cols = rng.integers(0, n, 6 * n)
        keep = rows != cols
        L = sp.csr_matrix((rng.uniform(0.0, 0.2, keep.sum()), (rows[keep], cols[keep])), shape=(n, n))
        L.sum_duplicates()
        L.sort_indices()
    zg = np.linspace(0.0, 3.0 * n_steps / 300.0, n_steps + 1)
    x0 = rng.uniform(0.5, 1.5, n)
    return d, L, zg, x0


def _device(a, dtype):
    import torch

    return torch.tensor(np.ascontiguousarray(a, dtype=dtype), device="cuda:0")


def _run_noalloc(ctx, d, L, zg, x0, calls=2, pass_indptr=True):
    import torch

    n = d.size
    td = _device(d, np.float64)
    tip = _device(L.indptr, np.int64)
    tix = _device(L.indices if L.nnz else np.zeros(1), np.int32)
    tv = _device(L.data if L.nnz else np.zeros(1), np.float64)
    tz = _device(zg, np.float64)
    outs = []
    for _ in range(calls):
        tx = _device(x0, np.float64)
        torch.cuda.synchronize()
        if pass_indptr:
            ctx.integrate_const_noalloc(n, td.data_ptr(), L.nnz, tip.data_ptr(), tix.data_ptr(), tv.data_ptr(),
                                        zg.size - 1, tz.data_ptr(), tx.data_ptr())
        else:
            ctx.integrate_const_noalloc(n, td.data_ptr(), 0, None, None, None, zg.size - 1, tz.data_ptr(),
                                        tx.data_ptr())
        outs.append(tx.cpu().numpy())
    return outs


@pytest.mark.parametrize("n,seed", [(3, 0), (5000, 1)])
def test_noalloc_matches_allocating_entry_point(n, seed):
    from prince_b200 import _lib

    ctx = _lib.Context(0)
    d, L, zg, x0 = _case(n, seed)
    ref = ctx.integrate_const(d, L, zg, x0)
    for out in _run_noalloc(ctx, d, L, zg, x0):
        np.testing.assert_allclose(out, ref, rtol=TOL, atol=0)


def test_noalloc_without_offdiagonal_entries():
    """nnz = 0 with NULL CSR pointers: the scratch's all-zero row pointer is used."""
    from prince_b200 import _lib

    ctx = _lib.Context(0)
    d, L, zg, x0 = _case(700, 2, offdiag=False)
    ref = ctx.integrate_const(d, None, zg, x0)
    np.testing.assert_allclose(ref, x0 * np.exp(d * (zg[-1] - zg[0])), rtol=1e-12)
    for out in _run_noalloc(ctx, d, L, zg, x0, pass_indptr=False):
        np.testing.assert_allclose(out, ref, rtol=TOL, atol=0)


def test_noalloc_zero_steps_leaves_the_state():
    from prince_b200 import _lib

    ctx = _lib.Context(0)
    d, L, zg, x0 = _case(257, 3, n_steps=0)
    assert zg.size == 1
    ref = ctx.integrate_const(d, L, zg, x0)
    np.testing.assert_array_equal(ref, x0)
    for out in _run_noalloc(ctx, d, L, zg, x0):
        np.testing.assert_array_equal(out, x0)


def test_noalloc_at_the_state_limit():
    """n = the static limit: every region of the scratch layout is used to its end."""
    from prince_b200 import _lib

    ctx = _lib.Context(0)
    d, L, zg, x0 = _case(MAX_STATES, 4, n_steps=12)
    ref = ctx.integrate_const(d, L, zg, x0)
    for out in _run_noalloc(ctx, d, L, zg, x0):
        np.testing.assert_allclose(out, ref, rtol=TOL, atol=0)


def test_noalloc_at_the_step_limit():
    from prince_b200 import _lib

    ctx = _lib.Context(0)
    d, L, zg, x0 = _case(64, 5, n_steps=MAX_STEPS)
    ref = ctx.integrate_const(d, L, zg, x0)
    for out in _run_noalloc(ctx, d, L, zg, x0, calls=1):
        np.testing.assert_allclose(out, ref, rtol=TOL, atol=0)


def test_noalloc_rejects_sizes_beyond_the_static_limit():
    from prince_b200 import _lib

    ctx = _lib.Context(0)
    buf = _device(np.zeros(4), np.float64)
    p = buf.data_ptr()
    with pytest.raises(ValueError, match="static scratch limit"):
        ctx.integrate_const_noalloc(MAX_STATES + 1, p, 0, None, None, None, 1, p, p)
    with pytest.raises(ValueError, match="static scratch limit"):
        ctx.integrate_const_noalloc(2, p, 0, None, None, None, MAX_STEPS + 1, p, p)


@pytest.mark.parametrize("defect", ["index_out_of_range", "negative_index", "indptr_decreasing", "indptr_end"])
def test_noalloc_rejects_malformed_csr_before_stepping(defect):
    """The device check reads only the declared sizes; nothing steps on a bad CSR,
    so the caller's state is left untouched, and a valid call afterwards is clean."""
    from prince_b200 import _lib

    ctx = _lib.Context(0)
    n = 6
    indptr = np.array([0, 1, 2, 3, 4, 5, 6], dtype=np.int64)
    indices = np.array([1, 2, 3, 4, 5, 0], dtype=np.int32)
    if defect == "index_out_of_range":
        indices[3] = n
    elif defect == "negative_index":
        indices[0] = -1
    elif defect == "indptr_decreasing":
        indptr[3] = 1
    else:
        indptr[-1] = 5
    nnz = 6
    vals = np.full(nnz, 0.1)
    d = np.full(n, -0.5)
    zg = np.linspace(0.0, 1.0, 11)
    x0 = np.arange(1.0, n + 1.0)
    td, tip, tix, tv, tz = (_device(d, np.float64), _device(indptr, np.int64), _device(indices, np.int32),
                            _device(vals, np.float64), _device(zg, np.float64))
    tx = _device(x0, np.float64)
    with pytest.raises(ValueError, match="CSR"):
        ctx.integrate_const_noalloc(n, td.data_ptr(), nnz, tip.data_ptr(), tix.data_ptr(), tv.data_ptr(),
                                    zg.size - 1, tz.data_ptr(), tx.data_ptr())
    np.testing.assert_array_equal(tx.cpu().numpy(), x0)
    d2, L2, zg2, x2 = _case(40, 6)
    ref = ctx.integrate_const(d2, L2, zg2, x2)
    np.testing.assert_allclose(_run_noalloc(ctx, d2, L2, zg2, x2, calls=1)[0], ref, rtol=TOL, atol=0)
