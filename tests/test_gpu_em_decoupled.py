"""Co-evolved EM cascade with gamma and e+- on a decoupled EM grid, on the device.

The reference run (``enable_em_decoupled_grid``: gamma and e+- in blocks of
the EM grid's bins ahead of the nuclei, ``core.py:105-137, 206-214``; the hooks
``_inject_bh_pairs`` / ``_apply_em_cascade`` with R_BH of shape EM grid x
nuclear grid) is pinned by ``light_network_em_decoupled.npz``.  The device
keeps the nuclei as bin-blocked species blocks and steps the EM rows as a
tail beside them; the states come back in the reference's layout.
"""

import numpy as np
import pytest

from golden_io import light_network_em_decoupled, rel_err_on_support
from oracle import etd2_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def em_golden():
    return light_network_em_decoupled()


def _blocks(run):
    return [s.sl for s in run.spec_man.species_refs]


def test_decoupled_single_rhs_matches_reference(em_golden):
    from prince_b200.solvers import UHECRPropagationSolverETD2
    z, run, em, source = em_golden
    s = UHECRPropagationSolverETD2(initial_z=0.2, final_z=0.0, prince_run=run)
    s.add_source_class(source("eq"))
    s.solve(dz=1e-3)
    assert rel_err_on_support(s.state, z["state_em"], _blocks(run)) < TOL
    E, g = s.res.get_solution(22)
    assert E.size == run.em_grid.d and np.array_equal(E, run.em_grid.grid)
    assert np.abs(g).max() > 0.0


def test_decoupled_multi_rhs_matches_reference(em_golden):
    from prince_b200 import _lib
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    z, run, em, source = em_golden
    m = MultiRHSPropagationSolverETD2(initial_z=0.2, final_z=0.0, prince_run=run, K=2)
    m[0].add_source_class(source("eq"))
    m[1].add_source_class(source("soft"))
    m.solve(dz=1e-3)
    assert rel_err_on_support(m.state, z["state_em_multi"], _blocks(run)) < TOL
    assert m._dev.ctx.info(_lib.PB_INFO_LAST_BLOCKED) == 1   # nuclei bin-blocked, EM rows as the tail


def test_decoupled_ragged_batch_vs_oracle(em_golden):
    """37 columns switching on at different redshifts, bin-blocked and general kernels."""
    from prince_b200 import _lib, cr_sources
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    z, run, em, source = em_golden
    rng = np.random.default_rng(12)
    K = 37
    cols = []
    for k in range(K):
        g = float(rng.uniform(1.0, 2.5))
        rc = float(10 ** rng.uniform(9.5, 11.0))
        frac = float(rng.uniform(0.2, 1.0))
        zmax = float(rng.uniform(0.05, 0.3))
        cols.append([cr_sources.RigdityCutoffSource(run, norm=1.0, params={2212: (g, rc, frac),
                                                                           1000020040: (g, rc, 1 - frac)},
                                                    z_max=zmax)])
    ref = O.OracleSolver(run, 0.3, 0.0, K=K, em=em, exp="cr").solve(cols, dz=1e-3)
    for mode in (1, 0):
        m = MultiRHSPropagationSolverETD2(initial_z=0.3, final_z=0.0, prince_run=run, K=K)
        m._dev.ctx.set_option(_lib.PB_OPT_BATCHED_KERNELS, mode)
        for k in range(K):
            m[k].add_source_class(cols[k][0])
        m.solve(dz=1e-3)
        m._dev.ctx.set_option(_lib.PB_OPT_BATCHED_KERNELS, 1)
        assert rel_err_on_support(m.state, ref, _blocks(run)) < TOL


def test_layout_rows_and_row_map_arguments():
    """The species-block / tail split and the caller row map, at the C ABI."""
    import scipy.sparse as sp
    from prince_b200 import _lib
    ctx = _lib.Context(0)
    n, d = 10, 4                      # two species blocks of 4 bins, two tail rows
    M = sp.lil_matrix((n, n))
    M[1, 5] = 1.0                     # block to block (bin-local)
    M[5, 1] = 1.0
    M = M.tocsr()
    ctx.set_coupling(n, M.indptr, M.indices)
    with pytest.raises(ValueError):
        ctx.set_layout(d, 9)          # not whole blocks
    with pytest.raises(ValueError):
        ctx.set_layout(d, 12)         # more block rows than states
    ctx.set_layout(d, 8)
    assert ctx.info(_lib.PB_INFO_BLOCKED_LAYOUT) in (0, 1)
    with pytest.raises(ValueError):
        ctx.set_row_map(np.array([0, 1, 2, 3, 4, 5, 6, 7, 8, 8]))   # not a permutation
    with pytest.raises(ValueError):
        ctx.set_row_map(np.array([0, 1, 2, 3, 4, 5, 6, 7, 8, 10]))  # out of range
    ctx.set_row_map(np.arange(n)[::-1].copy())
    ctx.set_row_map(None)
    # a coupling entry between the blocks and the tail keeps the general row kernels
    M2 = sp.lil_matrix((n, n))
    M2[9, 1] = 1.0
    M2 = M2.tocsr()
    ctx.set_coupling(n, M2.indptr, M2.indices)
    ctx.set_layout(d, 8)
    assert ctx.info(_lib.PB_INFO_BLOCKED_LAYOUT) == 0


def test_autotune_on_a_decoupled_em_solver(em_golden):
    """The stage autotuner runs on an EM solver (its short schedule carries its
    own EM windows) and the tuned solve still matches the reference."""
    import tempfile
    from prince_b200 import autotune
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    z, run, em, source = em_golden
    m = MultiRHSPropagationSolverETD2(initial_z=0.2, final_z=0.0, prince_run=run, K=2)
    m[0].add_source_class(source("eq"))
    m[1].add_source_class(source("soft"))
    with tempfile.TemporaryDirectory() as tdir:
        choice, cands = autotune.tune(m, path=tdir + "/autotune.json", force=True, steps=8, reps=1)
    assert cands and choice["steps_ms"] > 0
    m.solve(dz=1e-3)
    assert rel_err_on_support(m.state, z["state_em_multi"], _blocks(run)) < TOL
