"""Host-side construction of the constant operators of the ETD2 path.

* ``fd_loss_operator``: the finite-difference continuous-loss operator ``D``
  on a log-spaced grid, block-diagonal over species.  Rows use a 4th-order
  upwind-biased stencil on ln E with one-sided 3/4-point stencils in the
  first and last three rows, scaled by ``1/E_i`` -- the operator defined in
  ``src/prince_cr/solvers/partial_diff.py:48-110`` (block assembly
  ``partial_diff.py:28-46``).  The stencil table below is that operator's
  definition; the code that applies it is this package's own.
* ``split_diagonal``: ``(diag(L), L - diag(L))`` with explicit zeros removed
  and sorted columns, the contract of ``src/prince_cr/solvers/etd2.py:234-268``.
* ``coupling_structure``: the fixed CSR pattern of the photo-nuclear
  coupling matrix from the (daughter row, mother column) pairs of the fold
  kernel, with the kernel rows permuted into CSR order -- the contract of
  ``src/prince_cr/interaction_rates.py:648-697``.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .data import is_decoupled

# (first row, column offsets, integer weights, denominator) per stencil class.
_EDGE0 = ((1, 2, 3), (-3, 4, -1), 2.0)
_EDGE12 = ((-1, 0, 1, 2), (-2, -3, 6, -1), 6.0)
_BULK = ((-1, 0, 1, 2, 3), (-3, -10, 18, -6, 1), 12.0)


def _mirror(stencil):
    offs, w, den = stencil
    return tuple(-o for o in offs[::-1]), tuple(-c for c in w[::-1]), den


def fd_block(grid):
    """Dense ``(d, d)`` FD loss operator of one species block on ``grid``."""
    h = np.log(grid.bins[1] / grid.bins[0])
    d = grid.d
    last = d - 1
    op = np.zeros((d, d))

    def put(row, stencil):
        offs, w, den = stencil
        op[row, row + np.asarray(offs)] = np.asarray(w) / (den * h)

    put(0, _EDGE0)
    put(1, _EDGE12)
    put(2, _EDGE12)
    put(last, _mirror(_EDGE0))
    put(last - 1, _mirror(_EDGE12))
    put(last - 2, _mirror(_EDGE12))
    for row in range(3, d - 3):
        put(row, _BULK)
    return op * (1.0 / grid.grid)[:, None]


def fd_loss_operator(grid, nspec):
    """Block-diagonal CSR of ``nspec`` copies of ``fd_block(grid)``."""
    blk = sp.coo_matrix(fd_block(grid))
    return sp.block_diag(nspec * [blk]).tocsr()


def run_fd_loss_operator(run):
    """The run's FD loss operator: one block per species on its home grid, in
    ``princeidx`` order (``partial_diff.py:28-46``, heterogeneous path)."""
    sm = run.spec_man
    if not is_decoupled(sm):
        return fd_loss_operator(run.cr_grid, sm.nspec)
    cache = {}
    blocks = []
    for s in sorted(sm.species_refs, key=lambda x: x.princeidx):
        if s.grid_tag not in cache:
            cache[s.grid_tag] = sp.coo_matrix(fd_block(run.grids[s.grid_tag]))
        blocks.append(cache[s.grid_tag])
    return sp.block_diag(blocks).tocsr()


def split_diagonal(L):
    """``(d, L_off)``: float64 diagonal and the CSR off-diagonal part.

    Entries that are exactly zero after removing the diagonal are dropped and
    column indices are sorted within each row.
    """
    L = sp.csr_matrix(L)
    d = np.asarray(L.diagonal(), dtype=np.float64)
    off = (L - sp.diags(d, format="csr")).tocsr()
    off.eliminate_zeros()
    off.sort_indices()
    return d, off


def coupling_structure(rows, cols, n):
    """CSR pattern of the coupling matrix and the sort permutation.

    Returns ``(indptr, indices, order)`` where ``order`` sorts the kernel's
    (row, col) pairs into CSR order (rows, then columns).  Duplicated pairs
    are rejected: each fold-kernel row must own one matrix entry.
    """
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    order = np.lexsort((cols, rows))
    r = rows[order]
    c = cols[order]
    if r.size:
        if r[0] < 0 or r[-1] >= n or c.min() < 0 or c.max() >= n:
            raise ValueError("coupling entry outside the state vector")
        key = r * n + c
        if np.any(key[1:] == key[:-1]):
            raise ValueError("coupling pattern has duplicated (row, col) entries")
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=indptr[1:])
    return indptr, c.astype(np.int32), order
