"""Co-evolved EM cascade on the device against the reference and the oracle.

The reference run (``propagation.py:540-665``: ``_inject_bh_pairs`` then
``_apply_em_cascade`` after every ETD2 step) is pinned by the
``light_network_em.npz`` fixture; larger batches are checked against the
oracle's restatement of the same hook.
"""

import numpy as np
import pytest

from golden_io import light_network_em, rel_err_on_support
from oracle import etd2_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def em_golden():
    return light_network_em()


def _blocks(run):
    return [s.sl for s in run.spec_man.species_refs]


def test_em_cascade_single_rhs_matches_reference(em_golden):
    from prince_b200.solvers import UHECRPropagationSolverETD2
    z, run, em, source = em_golden
    s = UHECRPropagationSolverETD2(initial_z=0.2, final_z=0.0, prince_run=run)
    s.add_source_class(source("eq"))
    s.solve(dz=1e-3)
    assert rel_err_on_support(s.state, z["state_em"], _blocks(run)) < TOL
    g = run.spec_man.pdgid2sref[22].sl
    assert np.abs(s.state[g]).max() > 0.0   # the cascade fed the photons


def test_em_cascade_multi_rhs_matches_reference(em_golden):
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    z, run, em, source = em_golden
    m = MultiRHSPropagationSolverETD2(initial_z=0.2, final_z=0.0, prince_run=run, K=2)
    m[0].add_source_class(source("eq"))
    m[1].add_source_class(source("soft"))
    m.solve(dz=1e-3)
    assert rel_err_on_support(m.state, z["state_em_multi"], _blocks(run)) < TOL


def test_em_cascade_ragged_batch_vs_oracle(em_golden):
    """37 columns (a partial column tile) switching on at different redshifts."""
    from prince_b200 import cr_sources
    from prince_b200.solvers import MultiRHSPropagationSolverETD2
    z, run, em, source = em_golden
    rng = np.random.default_rng(11)
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
    m = MultiRHSPropagationSolverETD2(initial_z=0.3, final_z=0.0, prince_run=run, K=K)
    for k in range(K):
        m[k].add_source_class(cols[k][0])
    m.solve(dz=1e-3)
    ref = O.OracleSolver(run, 0.3, 0.0, K=K, em=em, exp="cr").solve(cols, dz=1e-3)
    assert rel_err_on_support(m.state, ref, _blocks(run)) < TOL


def test_em_cascade_adjoint_refuses_the_photon_scale_gradient(em_golden):
    """The transfer's dependence on the photon field is not differentiated."""
    import torch
    from prince_b200 import adjoint as AD
    z, run, em, source = em_golden
    sb = AD.SourceBatch(run, [2212], z_max=[0.1], initial_z=0.1)
    plan = sb.plan(0.1, ckpt_every=8)
    assert plan.em
    G = sb.grids(torch.tensor([2.0]), torch.tensor([10.0]), torch.tensor([[1.0]]))
    coeff = sb.coefficients(torch.tensor([0.0]))
    scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    X = AD.PropagateFunction.apply(G, coeff, scale, plan)
    X.sum().backward()
    assert scale.grad is None
